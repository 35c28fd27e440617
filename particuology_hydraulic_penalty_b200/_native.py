"""ctypes binding of libpscb200.so (the C ABI in ``include/psc_b200.h``).

This is the only module that talks to the shared library.  It fails loudly:
a missing or stale library raises ``NativeLibraryError``; every non-zero
status from the library raises ``PscError`` with the library's message.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_size_t, c_uint, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpscb200.so"
HEADER_PATH = Path(__file__).resolve().parents[1] / "include" / "psc_b200.h"

ABI_VERSION = 5

# status codes
PSC_OK = 0
PSC_E_INVALID = -1
PSC_E_CUDA = -2
PSC_E_UNSUPPORTED = -3
PSC_E_CAPACITY = -4

# storage modes
STORE_F64_EXACT = 0
STORE_F64 = 1
STORE_F32 = 2
STORE_F16 = 3
STORE_BF16 = 4

# step flags
STEP_COLLIDE = 1
STEP_IMB = 2
STEP_MOMENTS = 4
STEP_REDUCE = 8
STEP_MOVING = 16

WIN_MOVING = 1
WIN_INACTIVE = 2
WIN_OPEN_X = 4  # velocity inlet at x = 0, zero-gradient outflow at x = nx - 1

# reduction slots
RED_RHO, RED_UX, RED_UY, RED_UZ = 0, 1, 2, 3
RED_FLUID_UX, RED_FLUID_UY, RED_FLUID_UZ, RED_FLUID = 4, 5, 6, 7
RED_IMBX, RED_IMBY, RED_IMBZ = 8, 9, 10
RED_NONFINITE = 11
RED_SOLID = 12
NRED = 13
PARTIAL_ROWS = 8  # partial rows per tile (one per warp of a step CTA)

DIAG_MOMENTUM_RESIDUAL, DIAG_MAX_FORCE, DIAG_MAX_TORQUE = 0, 1, 2
DIAG_FORCE_SUM = (3, 4, 5)
NDIAG = 6

STEP_THREADS = 256
LOADS_STATIC_MAX_CHUNKS = 16384


class NativeLibraryError(RuntimeError):
    """libpscb200.so is missing, stale or not loadable."""


class PscError(RuntimeError):
    """A library call returned a non-zero status."""

    def __init__(self, code: int, func: str, message: str):
        super().__init__(f"{func} failed ({code}): {message}")
        self.code = code


class PscWindow(ctypes.Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("subsamples", c_int32), ("flags", c_int32), ("tile_cells", c_int32),
        ("tile_begin", c_int64), ("tile_count", c_int64),
        ("tau", c_double), ("force", c_double * 3), ("store_scale", c_double),
        ("f_src", c_void_p), ("f_dst", c_void_p), ("solid", c_void_p), ("level", c_void_p),
        ("us", c_void_p), ("imb", c_void_p), ("moments", c_void_p), ("partials", c_void_p),
        ("tau_minus", c_double), ("inlet_rho", c_double), ("inlet_u", c_double * 3),
    ]


class PscGeometry(ctypes.Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("subsamples", c_int32), ("nparticles", c_int32), ("chunk_entries", c_int32),
        ("capacity_entries", c_int64), ("capacity_chunks", c_int64),
        ("particles", c_void_p), ("bbox", c_void_p), ("ent_off", c_void_p), ("chunk_off", c_void_p),
        ("totals", c_void_p), ("ent_cnt", c_void_p), ("cell_n", c_void_p), ("cell_off", c_void_p),
        ("cl_pid", c_void_p), ("cl_cnt", c_void_p), ("alpha_sum", c_void_p), ("solid", c_void_p),
        ("level", c_void_p), ("scan_tmp", c_void_p),
        ("smooth_eps", c_double), ("ent_alpha", c_void_p), ("cl_ent", c_void_p),
        ("load_w", c_void_p), ("load_abk", c_void_p), ("load_n", c_void_p), ("list_ready", c_int32),
        ("reserved", c_int32),
    ]


class PscAdjointArgs(ctypes.Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("store", c_int32),
        ("tau", c_double), ("force", c_double * 3), ("kappa", c_double), ("dir", c_double * 3),
        ("state", c_void_p), ("solid", c_void_p), ("lam_in", c_void_p), ("lam_out", c_void_p),
        ("dKdB", c_void_p), ("dKdsolid", c_void_p),
    ]


KERNEL_AUTO, KERNEL_DIRECT, KERNEL_TMA, KERNEL_PAIR = 0, 1, 2, 3


class PscLaunch(ctypes.Structure):
    _fields_ = [("grid_ctas", c_int32), ("cells_per_thread", c_int32), ("kernel", c_int32), ("stages", c_int32),
                ("stage_bytes", c_int32)]


class PscConfig(ctypes.Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("subsamples", c_int32), ("store", c_int32),
        ("static_geometry", c_int32), ("device", c_int32), ("conv_min_steps", c_int32),
        ("tau", c_double), ("tau_minus", c_double), ("force", c_double * 3), ("store_scale", c_double),
        ("conv_tol", c_double), ("stream", c_void_p), ("open_x", c_int32), ("conv_check_every", c_int32),
        ("inlet_rho", c_double), ("inlet_u", c_double * 3),
    ]


class PscDiag(ctypes.Structure):
    _fields_ = [
        ("solid_volume_lu", c_double), ("mean_uz", c_double), ("momentum_residual", c_double),
        ("max_force", c_double), ("max_torque", c_double), ("mean_u", c_double * 3),
        ("superficial_u", c_double * 3), ("fluid_volume_lu", c_double), ("imb_sum", c_double * 3),
        ("force_sum", c_double * 3), ("permeability", c_double), ("nonfinite_cells", c_double),
    ]


class PscStatus(ctypes.Structure):
    _fields_ = [("steps_done", c_int32), ("converged", c_int32), ("residual", c_double), ("diag", PscDiag)]


# psc_step() flags and psc_get_fields() selectors
RUN_DIAG, RUN_CONVERGE, RUN_FIELDS = 1, 2, 4
FIELD_RHO, FIELD_UX, FIELD_UY, FIELD_UZ, FIELD_SOLID = 0, 1, 2, 3, 4
FIELD_IMB_X, FIELD_IMB_Y, FIELD_IMB_Z, FIELD_ALPHA_SUM = 5, 6, 7, 8
FIELD_US_X, FIELD_US_Y, FIELD_US_Z, FIELD_F = 9, 10, 11, 12

# name -> (restype, argtypes); every function of include/psc_b200.h
SIGNATURES = {
    "psc_abi_version": (c_int, []),
    "psc_last_error": (ctypes.c_char_p, []),
    "psc_window_size": (c_size_t, []),
    "psc_geometry_size": (c_size_t, []),
    "psc_adjoint_args_size": (c_size_t, []),
    "psc_scan_tmp_bytes": (c_size_t, [c_int64]),
    "psc_plan_tiles": (c_int, [POINTER(PscWindow), c_int, c_int, POINTER(c_int64)]),
    "psc_plan_row_tiles": (c_int, [POINTER(PscWindow), c_int, c_int, c_int, POINTER(c_int64), POINTER(c_int32)]),
    "psc_device_status": (c_int, [POINTER(c_int), c_int]),
    "psc_plan_pair_tiles": (c_int, [POINTER(PscWindow), c_int, POINTER(c_int64)]),
    "psc_init_equilibrium": (c_int, [c_int, c_double, c_void_p, c_int64, c_void_p]),
    "psc_geometry_plan": (c_int, [POINTER(PscGeometry), c_void_p]),
    "psc_geometry_build": (c_int, [POINTER(PscGeometry), c_void_p]),
    "psc_solid_velocity": (c_int, [POINTER(PscGeometry), c_int, c_void_p, c_void_p]),
    "psc_step_windows": (c_int, [c_int, c_void_p, c_int, c_int64, c_uint, c_int, c_void_p]),
    "psc_step_windows_ex": (c_int, [c_int, c_void_p, c_int, c_int64, c_uint, POINTER(PscLaunch), c_void_p]),
    "psc_reduce_windows": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "psc_particle_loads": (c_int, [POINTER(PscGeometry), c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p, c_void_p, c_void_p]),
    "psc_particle_loads_static": (c_int, [POINTER(PscGeometry), c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                          c_void_p, c_void_p]),
    "psc_adjoint_seed": (c_int, [POINTER(PscAdjointArgs), c_void_p]),
    "psc_adjoint_step": (c_int, [POINTER(PscAdjointArgs), c_void_p]),
    "psc_adjoint_geometry_grad": (c_int, [POINTER(PscGeometry), POINTER(PscAdjointArgs), c_void_p, c_void_p,
                                          c_void_p]),
    "psc_equilibrium": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p]),
    "psc_guo_force": (c_int, [c_double, c_double, c_double, c_void_p, c_void_p, c_void_p, c_double, c_void_p, c_int64,
                              c_void_p]),
    "psc_voxelize_spheres": (c_int, [c_void_p, c_int, POINTER(c_double), POINTER(c_double), c_double, c_int, c_int,
                                     c_int, c_void_p, c_void_p]),
    "psc_bounceback_step": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_double, c_double, c_double,
                                    c_double, c_uint, c_void_p, c_void_p]),
    "psc_stream_push": (c_int, [c_int, c_double, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p]),
    "psc_stream_pull_store": (c_int, [c_int, c_double, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p]),
    "psc_stream_push_open": (c_int, [c_int, c_double, c_void_p, c_void_p, c_int, c_int, c_int, c_double,
                                     POINTER(c_double), c_void_p]),
    "psc_stream_pull_store_open": (c_int, [c_int, c_double, c_void_p, c_void_p, c_int, c_int, c_int, c_double,
                                           POINTER(c_double), c_void_p]),
    # handle layer
    "psc_create": (c_int, [POINTER(PscConfig), POINTER(c_void_p)]),
    "psc_destroy": (c_int, [c_void_p]),
    "psc_set_particles": (c_int, [c_void_p, c_void_p, c_int]),
    "psc_rebuild_geometry": (c_int, [c_void_p]),
    "psc_step": (c_int, [c_void_p, c_int, c_uint, POINTER(PscStatus)]),
    "psc_converge": (c_int, [c_void_p, c_int, c_double, c_int, c_int, c_uint, POINTER(PscStatus)]),
    "psc_solver_last_error": (ctypes.c_char_p, [c_void_p]),
    "psc_batch_last_error": (ctypes.c_char_p, [c_void_p]),
    "psc_adjoint_last_error": (ctypes.c_char_p, [c_void_p]),
    "psc_get_fields": (c_int, [c_void_p, c_int, c_void_p]),
    "psc_set_populations": (c_int, [c_void_p, c_void_p]),
    "psc_get_loads": (c_int, [c_void_p, c_void_p, c_void_p]),
    "psc_get_diag": (c_int, [c_void_p, POINTER(PscDiag)]),
    "psc_accumulate_particle_loads": (c_int, [c_void_p]),
    "psc_get_sparse_alpha": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64]),
    "psc_solver_info": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int64)]),
    "psc_adjoint_create": (c_int, [POINTER(PscConfig), c_double, c_int, c_int, POINTER(c_void_p)]),
    "psc_adjoint_destroy": (c_int, [c_void_p]),
    "psc_adjoint_forward": (c_int, [c_void_p, c_void_p, c_int, POINTER(c_double)]),
    "psc_adjoint_backward": (c_int, [c_void_p, c_void_p]),
    "psc_config_size": (c_size_t, []),
    "psc_diag_size": (c_size_t, []),
    "psc_status_size": (c_size_t, []),
    "psc_batch_create": (c_int, [POINTER(PscConfig), c_int, POINTER(PscLaunch), c_int, POINTER(c_void_p)]),
    "psc_batch_destroy": (c_int, [c_void_p]),
    "psc_batch_set_particles": (c_int, [c_void_p, c_int, c_void_p, c_int]),
    "psc_batch_set_particles_all": (c_int, [c_void_p, POINTER(c_void_p), POINTER(c_int)]),
    "psc_batch_step": (c_int, [c_void_p, c_int, c_uint, POINTER(PscStatus)]),
    "psc_batch_converge": (c_int, [c_void_p, c_double, c_int, c_int, c_int, c_int, POINTER(PscStatus)]),
    "psc_batch_get_diag": (c_int, [c_void_p, c_int, POINTER(PscDiag)]),
    "psc_batch_get_loads": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "psc_batch_get_fields": (c_int, [c_void_p, c_int, c_int, c_void_p]),
}

_lib = None


def load(path: Path | None = None) -> ctypes.CDLL:
    """Load (once) and type the shared library; raise if it is absent or stale."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise NativeLibraryError(
            f"{p} not found: build it with `python -m particuology_hydraulic_penalty_b200.build`")
    try:
        lib = ctypes.CDLL(str(p))
    except OSError as exc:  # pragma: no cover - depends on the host
        raise NativeLibraryError(f"cannot load {p}: {exc}") from exc
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.psc_abi_version() != ABI_VERSION:
        raise NativeLibraryError("libpscb200.so ABI version mismatch: rebuild the library")
    if (lib.psc_window_size() != ctypes.sizeof(PscWindow) or lib.psc_geometry_size() != ctypes.sizeof(PscGeometry)
            or lib.psc_adjoint_args_size() != ctypes.sizeof(PscAdjointArgs)
            or lib.psc_config_size() != ctypes.sizeof(PscConfig) or lib.psc_diag_size() != ctypes.sizeof(PscDiag)
            or lib.psc_status_size() != ctypes.sizeof(PscStatus)):
        raise NativeLibraryError("libpscb200.so struct layout mismatch: rebuild the library")
    if path is None:
        _lib = lib
    return lib


def check(status: int, func: str) -> None:
    if status != PSC_OK:
        msg = load().psc_last_error()
        raise PscError(status, func, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    """Call a status-returning entry point and raise on failure."""
    check(getattr(load(), name)(*args), name)
