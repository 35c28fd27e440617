"""Python view of the handle layer of libpscb200.so (``psc_solver`` / ``psc_batch``).

The handles own their device memory, stream and CUDA graphs; everything
crossing this boundary is a NumPy host array.  One ``collide_stream_psc()``
step of the drop-in classes is one ``psc_step`` call here.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat

_VP = ctypes.c_void_p


def _addr(a: np.ndarray) -> int:
    # the array interface is much cheaper per call than ndarray.ctypes (which builds a helper object)
    return a.__array_interface__["data"][0]


def _ptr(a: np.ndarray):
    return _VP(_addr(a))


def _diag_dict(d: nat.PscDiag) -> dict:
    return {
        "solid_volume_lu": d.solid_volume_lu, "mean_uz": d.mean_uz, "momentum_residual": d.momentum_residual,
        "max_force": d.max_force, "max_torque": d.max_torque, "mean_u": tuple(d.mean_u),
        "superficial_u": tuple(d.superficial_u), "fluid_volume_lu": d.fluid_volume_lu, "imb_sum": tuple(d.imb_sum),
        "force_sum": tuple(d.force_sum), "permeability": d.permeability, "nonfinite_cells": d.nonfinite_cells,
    }


def make_config(shape, *, tau: float, force, subsamples: int, store: int, static_geometry: bool = True,
                device_index: int = 0, tau_minus: float = 0.0, store_scale: float | None = None,
                conv_tol: float = 0.0, conv_min_steps: int = 1, conv_check_every: int = 1,
                inlet=None) -> nat.PscConfig:
    c = nat.PscConfig()
    c.nx, c.ny, c.nz = (int(v) for v in shape)
    c.subsamples = int(subsamples)
    c.store = int(store)
    c.static_geometry = 1 if static_geometry else 0
    c.device = int(device_index)
    c.conv_min_steps = int(conv_min_steps)
    c.tau = float(tau)
    c.tau_minus = float(tau_minus)
    f = [float(v) for v in force]
    if len(f) != 3:
        raise ValueError("force must have three components")
    c.force[0], c.force[1], c.force[2] = f
    c.store_scale = 0.0 if store_scale is None else float(store_scale)
    c.conv_tol = float(conv_tol)
    c.conv_check_every = int(conv_check_every)
    c.stream = None
    if inlet is not None:  # (rho_in, (ux, uy, uz)): open along x
        c.open_x = 1
        c.inlet_rho = float(inlet[0])
        c.inlet_u[0], c.inlet_u[1], c.inlet_u[2] = (float(v) for v in inlet[1])
    return c


class SolverHandle:
    """One ``psc_solver``: a lattice window with its particles and results."""

    def __init__(self, cfg: nat.PscConfig):
        self._lib = nat.load()
        self.cfg = cfg
        self.shape = (cfg.nx, cfg.ny, cfg.nz)
        self.N = cfg.nx * cfg.ny * cfg.nz
        self._h = _VP()
        nat.call("psc_create", ctypes.byref(cfg), ctypes.byref(self._h))
        self._status = nat.PscStatus()
        self._step_fn = self._lib.psc_step
        self._set_fn = self._lib.psc_set_particles
        self.P = 0

    def close(self) -> None:
        if self._h is not None and self._h.value:
            self._lib.psc_destroy(self._h)
        self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, name: str) -> None:
        if rc != nat.PSC_OK:
            nat.check(rc, name)

    # particles and geometry -------------------------------------------------
    def set_particles(self, arr: np.ndarray) -> None:
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        self._check(self._set_fn(self._h, _ptr(arr), int(arr.shape[0])), "psc_set_particles")
        self.P = int(arr.shape[0])

    def rebuild_geometry(self) -> None:
        self._check(self._lib.psc_rebuild_geometry(self._h), "psc_rebuild_geometry")

    # stepping -----------------------------------------------------------------
    def step(self, nsteps: int = 1, flags: int = nat.RUN_DIAG) -> nat.PscStatus:
        st = self._status
        self._check(self._step_fn(self._h, int(nsteps), int(flags), ctypes.byref(st)), "psc_step")
        return st

    def converge(self, max_steps: int, tol: float = 1.0e-8, min_steps: int = 1, check_every: int = 1,
                 flags: int = 0) -> nat.PscStatus:
        """``psc_converge``: lbm_converge (couple_psc_liggghts.py:284-296) with the criterion on the device."""
        st = self._status
        self._check(self._lib.psc_converge(self._h, int(max_steps), float(tol), int(min_steps), int(check_every),
                                           int(flags), ctypes.byref(st)), "psc_converge")
        return st

    # results ------------------------------------------------------------------
    def field(self, which: int) -> np.ndarray:
        n = self.N * (19 if which == nat.FIELD_F else 1)
        out = np.empty(n, dtype=np.float64)
        self._check(self._lib.psc_get_fields(self._h, int(which), _ptr(out)), "psc_get_fields")
        return out

    def set_populations(self, f: np.ndarray) -> None:
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        if f.size != 19 * self.N:
            raise ValueError(f"f must have 19 x {self.shape} elements")
        self._check(self._lib.psc_set_populations(self._h, _ptr(f)), "psc_set_populations")

    def loads(self) -> tuple[np.ndarray, np.ndarray]:
        F = np.zeros((self.P, 3))
        T = np.zeros((self.P, 3))
        self._check(self._lib.psc_get_loads(self._h, _ptr(F), _ptr(T)), "psc_get_loads")
        return F, T

    def accumulate_loads(self) -> None:
        self._check(self._lib.psc_accumulate_particle_loads(self._h), "psc_accumulate_particle_loads")

    def diag(self) -> nat.PscDiag:
        d = nat.PscDiag()
        self._check(self._lib.psc_get_diag(self._h, ctypes.byref(d)), "psc_get_diag")
        return d

    def sparse_alpha(self) -> tuple[list, list]:
        """Per-particle ascending node ids and solid fractions (SparsePscD3Q19.node_ids / alpha_vals)."""
        P = self.P
        off = np.zeros(P + 1, dtype=np.int64)
        rc = self._lib.psc_get_sparse_alpha(self._h, _ptr(off), None, None, 0)
        if rc not in (nat.PSC_OK, nat.PSC_E_CAPACITY):
            self._check(rc, "psc_get_sparse_alpha")
        total = int(off[-1]) if P else 0
        ids = np.zeros(max(total, 1), dtype=np.int64)
        vals = np.zeros(max(total, 1))
        self._check(self._lib.psc_get_sparse_alpha(self._h, _ptr(off), _ptr(ids), _ptr(vals), total),
                    "psc_get_sparse_alpha")
        return ([ids[off[p]:off[p + 1]].copy() for p in range(P)], [vals[off[p]:off[p + 1]].copy() for p in range(P)])


class BatchHandle:
    """One ``psc_batch``: windows of uneven size stepped by one persistent launch per step."""

    def __init__(self, cfgs: list, launch: nat.PscLaunch | None = None, graph_steps: int = 20):
        self._lib = nat.load()
        self.nwin = len(cfgs)
        arr = (nat.PscConfig * self.nwin)(*cfgs)
        self.cells = np.array([c.nx * c.ny * c.nz for c in cfgs], dtype=np.int64)
        self.shapes = [(c.nx, c.ny, c.nz) for c in cfgs]
        self._h = _VP()
        nat.call("psc_batch_create", arr, self.nwin, ctypes.byref(launch) if launch is not None else None,
                 int(graph_steps), ctypes.byref(self._h))
        self._status = (nat.PscStatus * self.nwin)()
        self.P = [0] * self.nwin
        # pointer and count arrays of the last set_particles_all, kept while the caller passes the
        # same float64 C-contiguous array objects (their buffers cannot move while referenced here)
        self._staged = None

    def close(self) -> None:
        if self._h is not None and self._h.value:
            self._lib.psc_batch_destroy(self._h)
        self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def set_particles(self, k: int, arr: np.ndarray) -> None:
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        nat.check(self._lib.psc_batch_set_particles(self._h, int(k), _ptr(arr), int(arr.shape[0])),
                  "psc_batch_set_particles")
        self.P[k] = int(arr.shape[0])

    def set_particles_all(self, arrays) -> None:
        """Every window's (P_k, 10) particle array in one call (the contents are read every call)."""
        arrays = list(arrays)
        st = self._staged
        if st is not None and len(arrays) == len(st[0]) and all(a is b for a, b in zip(arrays, st[0])):
            ptrs, counts = st[1], st[2]
        else:
            arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in arrays]
            if len(arrs) != self.nwin:
                raise ValueError(f"expected {self.nwin} particle arrays")
            ptrs = (_VP * self.nwin)(*[_addr(a) if a.size else None for a in arrs])
            counts = (ctypes.c_int * self.nwin)(*[int(a.shape[0]) for a in arrs])
            # reuse only when the caller's own arrays were passed on (no converted copies)
            self._staged = (arrs, ptrs, counts) if all(a is b for a, b in zip(arrays, arrs)) else None
        nat.check(self._lib.psc_batch_set_particles_all(self._h, ptrs, counts), "psc_batch_set_particles_all")
        self.P = [int(c) for c in counts]

    def step(self, nsteps: int, flags: int = 0):
        nat.check(self._lib.psc_batch_step(self._h, int(nsteps), int(flags), self._status), "psc_batch_step")
        return self._status

    def converge(self, tol: float = 1e-8, check_every: int = 200, max_steps: int = 200000, min_steps: int = 0,
                 freeze: bool = True):
        nat.check(self._lib.psc_batch_converge(self._h, float(tol), int(check_every), int(max_steps), int(min_steps),
                                               1 if freeze else 0, self._status), "psc_batch_converge")
        return self._status

    def diag(self, k: int) -> nat.PscDiag:
        d = nat.PscDiag()
        nat.check(self._lib.psc_batch_get_diag(self._h, int(k), ctypes.byref(d)), "psc_batch_get_diag")
        return d

    def loads(self, k: int) -> tuple[np.ndarray, np.ndarray]:
        F = np.zeros((self.P[k], 3))
        T = np.zeros((self.P[k], 3))
        nat.check(self._lib.psc_batch_get_loads(self._h, int(k), _ptr(F), _ptr(T)), "psc_batch_get_loads")
        return F, T

    def field(self, k: int, which: int) -> np.ndarray:
        n = int(self.cells[k]) * (19 if which == nat.FIELD_F else 1)
        out = np.empty(n, dtype=np.float64)
        nat.check(self._lib.psc_batch_get_fields(self._h, int(k), int(which), _ptr(out)), "psc_batch_get_fields")
        return out


class AdjointHandle:
    """One ``psc_adjoint``: K of a static window and dK/d(x, y, z, r) of every particle (native runtime)."""

    def __init__(self, cfg: nat.PscConfig, smooth_eps: float = 0.05, steps: int = 2000, checkpoint_every: int = 100):
        self._lib = nat.load()
        self._h = _VP()
        nat.call("psc_adjoint_create", ctypes.byref(cfg), float(smooth_eps), int(steps), int(checkpoint_every),
                 ctypes.byref(self._h))
        self.P = 0

    def close(self) -> None:
        if self._h is not None and self._h.value:
            self._lib.psc_adjoint_destroy(self._h)
        self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def forward(self, particles: np.ndarray) -> float:
        arr = np.ascontiguousarray(particles, dtype=np.float64)
        K = ctypes.c_double(0.0)
        nat.check(self._lib.psc_adjoint_forward(self._h, _ptr(arr), int(arr.shape[0]), ctypes.byref(K)),
                  "psc_adjoint_forward")
        self.P = int(arr.shape[0])
        return float(K.value)

    def backward(self) -> np.ndarray:
        g = np.zeros((self.P, 4))
        nat.check(self._lib.psc_adjoint_backward(self._h, _ptr(g) if self.P else None), "psc_adjoint_backward")
        return g


diag_dict = _diag_dict
