"""Drop-in replacements for the reference's ``PscD3Q19`` / ``SparsePscD3Q19``.

Same constructor arguments, methods, attributes and diagnostics as
src/lbm_dem/psc3d.py (wangjianfttt/particuology_Hydraulic-penalty-), so that
the permeability probe (scripts/run_psc_permeability_resolution.py:127-143),
the coupled driver (coupling_sync/couple_psc_liggghts.py:582-607) and the
validation drivers run unchanged on one B200.  Every step runs in
libpscb200.so behind one native solver handle (``psc_solver``: device
memory, stream, geometry, results); one ``collide_stream_psc()`` is one
``psc_step`` call.  Attributes are host copies made on access.

Extra keyword-only arguments (absent from the reference):
    precision   "fp64-exact" (default: bit-identical to the reference),
                "fp64", "fp32", "fp16", "bf16" (deviation storage)
    force       body-force vector (fx, fy, fz); default (0, 0, body_force_z)
    store_scale scale of the FP16/BF16 stored deviations
    device      CUDA device
    collision   "bgk" (default, the reference) or "trt" (two relaxation times,
                magic parameter 3/16; deviation storage modes only)
    inlet       None (default: periodic, the reference) or (rho_in, (ux, uy, uz)):
                open along x with a velocity inlet at x = 0 and a zero-gradient
                outflow at x = n - 1 (y and z stay periodic)
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _native as nat
from .engine import check_inlet, particles_array, require_cuda, store_mode, trt_tau_minus
from .handle import SolverHandle, _diag_dict, make_config

# D3Q19 velocity set in the reference's index order (psc3d.py:17-43).
C = np.array(
    [[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
     [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1],
     [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1]],
    dtype=int,
)
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=float)
OPP = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17])
CS2 = 1.0 / 3.0


def _to_dev(a, dev):
    return torch.from_numpy(np.array(a, dtype=np.float64, order="C")).to(dev)  # writable copy


def equilibrium(rho, ux, uy, uz) -> np.ndarray:
    """Second-order D3Q19 equilibrium, (19, *shape) (psc3d.py:97-103), computed on the GPU in FP64."""
    dev = require_cuda()
    shape = np.shape(rho)
    n = int(np.prod(shape)) if shape else 1
    with torch.cuda.device(dev):
        args = [_to_dev(np.broadcast_to(a, shape), dev) for a in (rho, ux, uy, uz)]
        out = torch.empty(19 * n, dtype=torch.float64, device=dev)
        from .engine import stream_handle, vp

        nat.call("psc_equilibrium", *(vp(a) for a in args), vp(out), n, stream_handle(dev))
        return out.view(19, *shape).cpu().numpy()


def guo_force(fx: float, fy: float, fz: float, ux, uy, uz, tau: float) -> np.ndarray:
    """Guo forcing term, (19, *shape) (psc3d.py:106-114), computed on the GPU in FP64."""
    dev = require_cuda()
    shape = np.shape(ux)
    n = int(np.prod(shape)) if shape else 1
    with torch.cuda.device(dev):
        args = [_to_dev(np.broadcast_to(a, shape), dev) for a in (ux, uy, uz)]
        out = torch.empty(19 * n, dtype=torch.float64, device=dev)
        from .engine import stream_handle, vp

        nat.call("psc_guo_force", float(fx), float(fy), float(fz), *(vp(a) for a in args), float(tau), vp(out), n,
                 stream_handle(dev))
        return out.view(19, *shape).cpu().numpy()


@dataclass
class Particle3D:
    """Sphere state in lattice units (psc3d.py:46-57)."""

    x: float
    y: float
    z: float
    r: float
    vx: float = 0.0
    vy: float = 0.0
    vz: float = 0.0
    wx: float = 0.0
    wy: float = 0.0
    wz: float = 0.0


class PscD3Q19:
    """D3Q19 PSC-IMB solver with node-summed particle loads (psc3d.py:117-281), on the GPU."""

    def __init__(self, n: int, particles, tau: float = 0.72, subsamples: int = 4, body_force_z: float = 0.0,
                 static_geometry: bool = False, *, precision: str = "fp64-exact", force=None,
                 store_scale: float | None = None, device=None, collision: str = "bgk", inlet=None):
        self._device = require_cuda(device)
        self.n = int(n)
        if self.n <= 0:
            raise ValueError("n must be positive")
        self.particles = particles
        self.tau = float(tau)
        self.subsamples = int(subsamples)
        self.body_force_z = float(body_force_z)
        self.static_geometry = bool(static_geometry)
        self.precision = precision
        self._store = store_mode(precision)
        self.force = (0.0, 0.0, self.body_force_z) if force is None else tuple(float(v) for v in force)
        if len(self.force) != 3:
            raise ValueError("force must have three components")
        if collision not in ("bgk", "trt"):
            raise ValueError("collision must be 'bgk' (the reference) or 'trt'")
        if collision == "trt" and self._store == nat.STORE_F64_EXACT:
            raise ValueError("TRT collision runs in the deviation storage modes (fp64, fp32, fp16, bf16)")
        if self._store != nat.STORE_F64_EXACT and self.subsamples ** 3 > 255:
            raise ValueError("the FP32/FP16/BF16 and fast-FP64 modes store the solid level as uint8 "
                             "and need subsamples <= 6")
        if store_scale is not None and not (np.isfinite(store_scale) and store_scale > 0.0):
            raise ValueError("store_scale must be a positive finite number")
        self.collision = collision
        self.inlet = check_inlet(inlet)
        index = self._device.index if self._device.index is not None else torch.cuda.current_device()
        cfg = make_config((self.n,) * 3, tau=self.tau, force=self.force, subsamples=self.subsamples,
                          store=self._store, static_geometry=self.static_geometry, device_index=index,
                          tau_minus=trt_tau_minus(self.tau) if collision == "trt" else 0.0, store_scale=store_scale,
                          inlet=self.inlet)
        self._h = SolverHandle(cfg)
        parr = particles_array(particles)
        self._h.set_particles(parr)
        self._P = parr.shape[0]
        self._geometry_built = False
        self._stepped = False
        self._loads_host = None
        self._cache: dict = {}
        self._hf = np.zeros((self._P, 3), dtype=float)
        self._ht = np.zeros((self._P, 3), dtype=float)
        self._momentum_residual = 0.0
        self._nonfinite = False

    # ------------------------------------------------------------------
    # geometry
    # ------------------------------------------------------------------
    def _upload_particles(self) -> None:
        parr = particles_array(self.particles)
        self._h.set_particles(parr)
        self._P = parr.shape[0]

    def rebuild_geometry(self) -> None:
        """Solid fraction from S^3 sub-samples per cell (psc3d.py:151-179 / 328-345)."""
        self._upload_particles()
        self._h.rebuild_geometry()
        self._geometry_built = True
        for key in ("solid", "sparse", "dense", "alpha_sum"):
            self._cache.pop(key, None)

    def solid_velocity(self):
        """alpha-weighted rigid-body velocity per node (psc3d.py:181-206 / 347-373)."""
        self._upload_particles()
        shape = self._shape3()
        us = [self._h.field(nat.FIELD_US_X + k).reshape(shape) for k in range(3)]
        self._geometry_built = True
        return us[0], us[1], us[2]

    # ------------------------------------------------------------------
    # the step
    # ------------------------------------------------------------------
    def collide_stream_psc(self) -> dict:
        """One PSC-IMB collide + stream step (psc3d.py:208-253)."""
        # positions / velocities may have been mutated in place: they feed the
        # geometry, the solid velocity and the torque arms (re-read every call)
        self._upload_particles()
        d = self._h.step(1, nat.RUN_DIAG).diag
        self._geometry_built = True
        self._stepped = True
        self._loads_host = None
        self._cache.clear()
        self._momentum_residual = float(d.momentum_residual)
        if d.nonfinite_cells > 0:
            self._nonfinite = True
        return {
            "solid_volume_lu": float(d.solid_volume_lu),
            "mean_uz": float(d.mean_uz),
            "momentum_residual": float(d.momentum_residual),
            "max_force": float(d.max_force),
            "max_torque": float(d.max_torque),
        }

    def advance(self, steps: int) -> dict:
        """``steps`` collide_stream_psc() steps in one native call, with the loads and diagnostics of
        the last one (the populations are those of ``steps`` single calls; the steps before the last
        take no reductions or loads).  Returns the last step's diagnostics dictionary."""
        steps = int(steps)
        if steps < 1:
            raise ValueError("steps must be >= 1")
        if steps == 1:
            return self.collide_stream_psc()
        self._upload_particles()
        d = self._h.step(steps, nat.RUN_DIAG).diag
        self._geometry_built = True
        self._stepped = True
        self._loads_host = None
        self._cache.clear()
        self._momentum_residual = float(d.momentum_residual)
        if d.nonfinite_cells > 0:
            self._nonfinite = True
        return {"solid_volume_lu": float(d.solid_volume_lu), "mean_uz": float(d.mean_uz),
                "momentum_residual": float(d.momentum_residual), "max_force": float(d.max_force),
                "max_torque": float(d.max_torque)}

    def step_diagnostics(self) -> dict:
        """Every diagnostic of the last step: the reference's five keys plus the Darcy quantities
        (mean and superficial velocity, fluid volume, IMB and force sums, permeability along the body
        force, non-finite cell count).  No GPU work: the values were taken with the step."""
        return _diag_dict(self._h.diag())

    def run_to_convergence(self, residual_tol: float = 1.0e-8, min_steps: int = 1, max_steps: int = 20000,
                           check_every: int = 1):
        """lbm_converge (coupling_sync/couple_psc_liggghts.py:284-296) as one native call.

        Steps until |mean_uz_k - mean_uz_{k-1}| / |mean_uz_k| < residual_tol at a step
        k >= min_steps, at most max_steps steps; returns (iterations, residual, converged,
        diagnostics of the last step) like the reference's loop.  The criterion is evaluated on the
        device; the loads and diagnostics are taken for the stopping step only.  check_every = 1
        evaluates it every step (the reference's iterations and residual); check_every = k evaluates
        it on steps k - 1 and k of every k, with no reductions on the steps in between.
        """
        self._upload_particles()
        st = self._h.converge(int(max_steps), float(residual_tol), int(min_steps), int(check_every))
        d = st.diag
        self._geometry_built = True
        self._stepped = True
        self._loads_host = None
        self._cache.clear()
        self._momentum_residual = float(d.momentum_residual)
        if d.nonfinite_cells > 0:
            self._nonfinite = True
        diag = {
            "solid_volume_lu": float(d.solid_volume_lu),
            "mean_uz": float(d.mean_uz),
            "momentum_residual": float(d.momentum_residual),
            "max_force": float(d.max_force),
            "max_torque": float(d.max_torque),
        }
        return int(st.steps_done), float(st.residual), bool(st.converged), diag

    # loads are copied to the host when read ------------------------------
    def _fetch_loads(self) -> None:
        if self._loads_host is None:
            f, t = self._h.loads()
            self._store_loads(f, t)
            self._loads_host = True

    @property
    def hydro_forces(self) -> np.ndarray:
        if self._stepped:
            self._fetch_loads()
        return self._hf

    @hydro_forces.setter
    def hydro_forces(self, value) -> None:
        if self._stepped:
            self._fetch_loads()  # results of the last step go into the old array first
        self._hf = value

    @property
    def hydro_torques(self) -> np.ndarray:
        if self._stepped:
            self._fetch_loads()
        return self._ht

    @hydro_torques.setter
    def hydro_torques(self, value) -> None:
        if self._stepped:
            self._fetch_loads()
        self._ht = value

    @property
    def momentum_residual(self) -> float:
        return self._momentum_residual

    @momentum_residual.setter
    def momentum_residual(self, value) -> None:
        self._momentum_residual = float(value)

    def _store_loads(self, forces: np.ndarray, torques: np.ndarray) -> None:
        # the coupled driver reallocates hydro_forces / hydro_torques itself
        # (couple_psc_liggghts.py:592-594); write into its arrays when they fit
        for name, val in (("_hf", forces), ("_ht", torques)):
            cur = getattr(self, name, None)
            if isinstance(cur, np.ndarray) and cur.shape == val.shape and cur.dtype == np.float64:
                cur[...] = val
            else:
                setattr(self, name, val.copy())

    def accumulate_particle_loads(self) -> None:
        """Recompute particle force / torque from the last step's IMB field (psc3d.py:255-281)."""
        if not self._stepped:
            # no IMB momentum yet: the loads of a fluid at rest are zero
            self._store_loads(np.zeros((self._P, 3)), np.zeros((self._P, 3)))
            self.momentum_residual = 0.0
            return
        self._upload_particles()
        self._h.accumulate_loads()
        f, t = self._h.loads()
        self._store_loads(f, t)
        self._loads_host = True
        self.momentum_residual = float(self._h.diag().momentum_residual)

    # ------------------------------------------------------------------
    # host views
    # ------------------------------------------------------------------
    def _shape3(self):
        return (self.n, self.n, self.n)

    def _field(self, which: int) -> np.ndarray:
        key = ("field", which)
        if key not in self._cache:
            self._cache[key] = self._h.field(which).reshape(self._shape3())
        return self._cache[key]

    @property
    def rho(self) -> np.ndarray:
        return self._field(nat.FIELD_RHO)

    @property
    def ux(self) -> np.ndarray:
        return self._field(nat.FIELD_UX)

    @property
    def uy(self) -> np.ndarray:
        return self._field(nat.FIELD_UY)

    @property
    def uz(self) -> np.ndarray:
        return self._field(nat.FIELD_UZ)

    @property
    def imb_mx(self) -> np.ndarray:
        return self._field(nat.FIELD_IMB_X)

    @property
    def imb_my(self) -> np.ndarray:
        return self._field(nat.FIELD_IMB_Y)

    @property
    def imb_mz(self) -> np.ndarray:
        return self._field(nat.FIELD_IMB_Z)

    @property
    def solid(self) -> np.ndarray:
        if "solid" not in self._cache:
            self._cache["solid"] = self._h.field(nat.FIELD_SOLID).reshape(self._shape3())
        return self._cache["solid"]

    @property
    def f(self) -> np.ndarray:
        """Post-stream populations (19, n, n, n), absolute FP64 (psc3d.py:140, :242)."""
        if "f" not in self._cache:
            self._cache["f"] = self._h.field(nat.FIELD_F).reshape((19, *self._shape3()))
        return self._cache["f"]

    @f.setter
    def f(self, value) -> None:
        self._h.set_populations(np.asarray(value, dtype=np.float64))
        self._cache.clear()

    def _sparse(self):
        if "sparse" not in self._cache:
            self._cache["sparse"] = self._h.sparse_alpha()
        return self._cache["sparse"]

    def _alpha_sum(self) -> np.ndarray:
        if "alpha_sum" not in self._cache:
            self._cache["alpha_sum"] = self._h.field(nat.FIELD_ALPHA_SUM)
        return self._cache["alpha_sum"]

    @property
    def alpha_p(self) -> np.ndarray:
        """Dense (P, n, n, n) solid fractions per particle (psc3d.py:141, :173)."""
        if "dense" not in self._cache:
            ids, vals = self._sparse()
            out = np.zeros((self._h.P, self.n ** 3))
            for p, (i, v) in enumerate(zip(ids, vals)):
                out[p, i] = v
            self._cache["dense"] = out.reshape((self._h.P, *self._shape3()))
        return self._cache["dense"]

    @property
    def owner_weights(self) -> np.ndarray:
        """alpha_p / sum alpha where the sum exceeds 1e-14 (psc3d.py:176-178)."""
        a = self.alpha_p
        s = self._alpha_sum().reshape(self._shape3())
        out = np.zeros_like(a)
        mask = s > 1.0e-14
        out[:, mask] = a[:, mask] / s[mask]
        return out


class SparsePscD3Q19(PscD3Q19):
    """Sparse PSC-IMB variant for packed-bed windows (psc3d.py:284-407), on the GPU.

    The GPU geometry is sparse for both classes (per-particle bounding-box
    entries and per-cell particle lists), so the two differ only in their
    defaults and in the host views they expose.  ``geometry_workers`` is
    accepted for call compatibility; voxelisation runs on the GPU.
    """

    def __init__(self, n: int, particles, tau: float = 0.72, subsamples: int = 3, body_force_z: float = 0.0,
                 static_geometry: bool = False, geometry_workers: int = 1, **kwargs):
        super().__init__(n, particles, tau=tau, subsamples=subsamples, body_force_z=body_force_z,
                         static_geometry=static_geometry, **kwargs)
        self.geometry_workers = max(1, int(geometry_workers))

    @property
    def node_ids(self) -> list:
        return self._sparse()[0]

    @property
    def alpha_vals(self) -> list:
        return self._sparse()[1]

    @property
    def alpha_sum_flat(self) -> np.ndarray:
        return self._alpha_sum()
