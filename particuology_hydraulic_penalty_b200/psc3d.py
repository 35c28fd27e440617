"""Drop-in replacements for the reference's ``PscD3Q19`` / ``SparsePscD3Q19``.

Same constructor arguments, methods, attributes and diagnostics as
src/lbm_dem/psc3d.py (wangjianfttt/particuology_Hydraulic-penalty-), so that
the permeability probe (scripts/run_psc_permeability_resolution.py:127-143),
the coupled driver (coupling_sync/couple_psc_liggghts.py:582-607) and the
validation drivers run unchanged on one B200.  Every step runs in
libpscb200.so; attributes are host copies made on access.

Extra keyword-only arguments (absent from the reference):
    precision   "fp64-exact" (default: bit-identical to the reference),
                "fp64", "fp32", "fp16", "bf16" (deviation storage)
    force       body-force vector (fx, fy, fz); default (0, 0, body_force_z)
    store_scale scale of the FP16/BF16 stored deviations
    device      CUDA device
    collision   "bgk" (default, the reference) or "trt" (two relaxation times,
                magic parameter 3/16; deviation storage modes only)
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _native as nat
from .engine import (DeviceGeometry, LatticeWindow, particles_array, require_cuda, store_mode, trt_tau_minus)

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
                 store_scale: float | None = None, device=None, collision: str = "bgk"):
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
        self.collision = collision
        shape = (self.n,) * 3
        with torch.cuda.device(self._device):
            self._win = LatticeWindow(shape, self.tau, self.force, self.subsamples, self._store, store_scale,
                                      self._device,
                                      tau_minus=trt_tau_minus(self.tau) if collision == "trt" else 0.0)
            self._geo = DeviceGeometry(shape, self.subsamples, self._device,
                                       want_level=self._store != nat.STORE_F64_EXACT)
            self._win.bind_geometry(self._geo)
            self._win.ensure_fields(imb=True, moments=True)
            parr = particles_array(particles)
            self._geo.set_particles(parr)
            self._P = parr.shape[0]
            self._forces_dev = torch.zeros((self._P, 3), dtype=torch.float64, device=self._device)
            self._torques_dev = torch.zeros((self._P, 3), dtype=torch.float64, device=self._device)
            # post-stream reductions and load diagnostics land in one buffer read back per call
            self._out_dev = torch.zeros(nat.NRED + nat.NDIAG, dtype=torch.float64, device=self._device)
            self._red_post_dev = self._out_dev[: nat.NRED]
            self._diag_dev = self._out_dev[nat.NRED:]
            self._out_host = torch.zeros(nat.NRED + nat.NDIAG, dtype=torch.float64).pin_memory()
        self._geometry_built = False
        self._stepped = False
        self._moments_ready = False
        self._loads_host = None
        self._cache: dict = {}
        self._hf = np.zeros((self._P, 3), dtype=float)
        self._ht = np.zeros((self._P, 3), dtype=float)
        self._momentum_residual = 0.0

    # ------------------------------------------------------------------
    # geometry
    # ------------------------------------------------------------------
    def _upload_particles(self) -> np.ndarray:
        parr = particles_array(self.particles)
        with torch.cuda.device(self._device):
            self._geo.set_particles(parr)
            if parr.shape[0] != self._P:
                self._P = parr.shape[0]
                self._forces_dev = torch.zeros((self._P, 3), dtype=torch.float64, device=self._device)
                self._torques_dev = torch.zeros((self._P, 3), dtype=torch.float64, device=self._device)
                self._geometry_built = False
        return parr

    def rebuild_geometry(self) -> None:
        """Solid fraction from S^3 sub-samples per cell (psc3d.py:151-179 / 328-345)."""
        self._upload_particles()
        with torch.cuda.device(self._device):
            self._geo.rebuild()
        self._geometry_built = True
        self._cache.pop("solid", None)
        self._cache.pop("dense", None)
        self._cache.pop("sparse", None)

    def solid_velocity(self):
        """alpha-weighted rigid-body velocity per node (psc3d.py:181-206 / 347-373)."""
        if not self._geometry_built:
            self.rebuild_geometry()
        with torch.cuda.device(self._device):
            us = torch.empty(3 * self._geo.N, dtype=torch.float64, device=self._device)
            self._geo.solid_velocity(us)
            us = us.view(3, self.n, self.n, self.n).cpu().numpy()
        return us[0], us[1], us[2]

    # ------------------------------------------------------------------
    # the step
    # ------------------------------------------------------------------
    def collide_stream_psc(self) -> dict:
        """One PSC-IMB collide + stream step (psc3d.py:208-253)."""
        with torch.cuda.device(self._device):
            if (not self.static_geometry) or (not self._geometry_built):
                self.rebuild_geometry()
            else:
                # positions / velocities may have been mutated in place: they feed
                # the solid velocity and the torque arms even for static geometry
                self._upload_particles()
                if not self._geometry_built:
                    self.rebuild_geometry()
            parr = self._geo.host_particles
            moving = bool(parr.shape[0]) and bool(np.any(parr[:, 4:10] != 0.0))
            win = self._win
            if moving:
                self._geo.solid_velocity(win.ensure_us())
            win.set_moving(moving)
            win.step(nat.STEP_IMB | nat.STEP_REDUCE)
            win.reduce(win.red)
            self._geo.loads(win.imb, win.red[nat.RED_IMBX:], self._forces_dev, self._torques_dev, self._diag_dev)
            # reductions of the post-stream state only; the fields are made on access
            win.moments_pass(self._red_post_dev, write_fields=False)
            self._out_host.copy_(self._out_dev, non_blocking=True)
            torch.cuda.current_stream(self._device).synchronize()
        self._stepped = True
        self._moments_ready = False
        self._loads_host = None
        self._cache.clear()
        host = self._out_host.numpy()
        red_post = host[: nat.NRED]
        diag = host[nat.NRED:]
        P = self._P
        self._momentum_residual = float(diag[nat.DIAG_MOMENTUM_RESIDUAL])
        if red_post[nat.RED_NONFINITE] > 0:
            self._nonfinite = True
        return {
            "solid_volume_lu": float(red_post[nat.RED_SOLID]),
            "mean_uz": float(red_post[nat.RED_UZ] / self._geo.N),
            "momentum_residual": float(self._momentum_residual),
            "max_force": float(diag[nat.DIAG_MAX_FORCE]) if P else 0.0,
            "max_torque": float(diag[nat.DIAG_MAX_TORQUE]) if P else 0.0,
        }

    # loads are copied to the host when read ------------------------------
    def _fetch_loads(self) -> None:
        if self._loads_host is None:
            with torch.cuda.device(self._device):
                f = self._forces_dev.cpu().numpy()
                t = self._torques_dev.cpu().numpy()
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
        if not self._geometry_built:
            self.rebuild_geometry()
        with torch.cuda.device(self._device):
            self._geo.loads(self._win.imb, self._win.red[nat.RED_IMBX:], self._forces_dev, self._torques_dev,
                            self._diag_dev)
            host = torch.cat([self._diag_dev, self._forces_dev.view(-1), self._torques_dev.view(-1)]).cpu().numpy()
        P = self._P
        self._store_loads(host[nat.NDIAG: nat.NDIAG + 3 * P].reshape(P, 3), host[nat.NDIAG + 3 * P:].reshape(P, 3))
        self._loads_host = True
        self.momentum_residual = float(host[nat.DIAG_MOMENTUM_RESIDUAL])

    # ------------------------------------------------------------------
    # host views
    # ------------------------------------------------------------------
    def _shape3(self):
        return (self.n, self.n, self.n)

    def _moment(self, k: int) -> np.ndarray:
        if not self._stepped:
            return np.ones(self._shape3()) if k == 0 else np.zeros(self._shape3())
        if not self._moments_ready:
            with torch.cuda.device(self._device):
                self._win.moments_pass(None, write_fields=True)
            self._moments_ready = True
        key = ("mom", k)
        if key not in self._cache:
            N = self._geo.N
            self._cache[key] = self._win.moments[k * N:(k + 1) * N].to(torch.float64).cpu().numpy().reshape(
                self._shape3())
        return self._cache[key]

    @property
    def rho(self) -> np.ndarray:
        return self._moment(0)

    @property
    def ux(self) -> np.ndarray:
        return self._moment(1)

    @property
    def uy(self) -> np.ndarray:
        return self._moment(2)

    @property
    def uz(self) -> np.ndarray:
        return self._moment(3)

    def _imb(self, k: int) -> np.ndarray:
        key = ("imb", k)
        if key not in self._cache:
            N = self._geo.N
            self._cache[key] = self._win.imb[k * N:(k + 1) * N].to(torch.float64).cpu().numpy().reshape(
                self._shape3())
        return self._cache[key]

    @property
    def imb_mx(self) -> np.ndarray:
        return self._imb(0)

    @property
    def imb_my(self) -> np.ndarray:
        return self._imb(1)

    @property
    def imb_mz(self) -> np.ndarray:
        return self._imb(2)

    @property
    def solid(self) -> np.ndarray:
        if not self._geometry_built:
            return np.zeros(self._shape3())
        if "solid" not in self._cache:
            self._cache["solid"] = self._geo.solid.cpu().numpy().reshape(self._shape3())
        return self._cache["solid"]

    @property
    def f(self) -> np.ndarray:
        """Post-stream populations (19, n, n, n), absolute FP64 (psc3d.py:140, :242)."""
        if "f" not in self._cache:
            with torch.cuda.device(self._device):
                self._cache["f"] = self._win.post_stream_f().cpu().numpy()
        return self._cache["f"]

    @f.setter
    def f(self, value) -> None:
        t = torch.as_tensor(np.asarray(value, dtype=np.float64))
        with torch.cuda.device(self._device):
            self._win.load_post_stream_f(t)
        self._cache.clear()
        self._moments_ready = False

    @property
    def alpha_p(self) -> np.ndarray:
        """Dense (P, n, n, n) solid fractions per particle (psc3d.py:141, :173)."""
        if "dense" not in self._cache:
            ids, vals = self._geo.sparse_lists() if self._geometry_built else ([], [])
            n3 = self._geo.N
            out = np.zeros((self._P, n3))
            for p, (i, v) in enumerate(zip(ids, vals)):
                out[p, i] = v
            self._cache["dense"] = out.reshape((self._P, *self._shape3()))
        return self._cache["dense"]

    @property
    def owner_weights(self) -> np.ndarray:
        """alpha_p / sum alpha where the sum exceeds 1e-14 (psc3d.py:176-178)."""
        a = self.alpha_p
        s = self._geo.alpha_sum.cpu().numpy().reshape(self._shape3()) if self._geometry_built else np.zeros(
            self._shape3())
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

    def _sparse(self):
        if "sparse" not in self._cache:
            self._cache["sparse"] = self._geo.sparse_lists() if self._geometry_built else ([], [])
        return self._cache["sparse"]

    @property
    def node_ids(self) -> list:
        return self._sparse()[0]

    @property
    def alpha_vals(self) -> list:
        return self._sparse()[1]

    @property
    def alpha_sum_flat(self) -> np.ndarray:
        if not self._geometry_built:
            return np.zeros(self._geo.N)
        return self._geo.alpha_sum.cpu().numpy()
