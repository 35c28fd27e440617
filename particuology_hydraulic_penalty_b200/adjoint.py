"""d(permeability)/d(particle centres, radii) by a hand-written adjoint.

``PermeabilityProblem`` runs one static periodic window forward (smooth
sub-sampled solid fraction, deviation storage in FP32 or FP64, checkpoints
every ``checkpoint_every`` steps) and backward (segment recomputation from
the checkpoints, then reverse steps with ``psc_adjoint_step``), giving
dK/d(x, y, z, r) for every particle.  ``permeability(centres, radii,
problem)`` wraps it as a ``torch.autograd.Function``.

The reference's solid fraction counts inside sub-samples
(src/lbm_dem/psc3d.py:79-90) and is piecewise constant in the particle
state, so its derivative is zero almost everywhere; the adjoint
differentiates the smooth surrogate in which each sample contributes
sigma((r - d) / eps).  ``solid_gap()`` reports how far that surrogate is from
the counted solid fraction of the same particles.

Cost: forward T steps + recomputation T steps + T reverse steps, each
reverse step moving ~1.6x the bytes of a forward step.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native as nat
from .engine import DeviceGeometry, LatticeWindow, particles_array, require_cuda, store_mode, stream_handle, \
    struct_to_device, vp

Q = 19


class PermeabilityProblem:
    """K of one static window and its adjoint gradient w.r.t. every particle's (x, y, z, r)."""

    def __init__(self, n: int, tau: float = 0.8, force=(1.0e-6, 0.0, 0.0), subsamples: int = 4,
                 eps: float = 0.05, steps: int = 2000, checkpoint_every: int = 100, precision: str = "fp32",
                 device=None):
        self.device = require_cuda(device)
        self.n = int(n)
        self.N = self.n ** 3
        self.tau = float(tau)
        self.force = tuple(float(v) for v in force)
        self.fmag = float(np.linalg.norm(self.force))
        if self.fmag <= 0.0:
            raise ValueError("the permeability needs a non-zero body force")
        self.dir = tuple(v / self.fmag for v in self.force)
        self.subsamples = int(subsamples)
        self.eps = float(eps)
        self.steps = int(steps)
        self.every = int(checkpoint_every)
        if self.steps < 1 or self.every < 1:
            raise ValueError("steps and checkpoint_every must be >= 1")
        self.store = store_mode(precision)
        if self.store not in (nat.STORE_F32, nat.STORE_F64):
            raise ValueError("the adjoint runs in the fp32 or fp64 deviation modes")
        self.nu = (self.tau - 0.5) / 3.0
        self.kappa = self.nu / (self.fmag * self.N)
        self._fdtype = torch.float64 if self.store == nat.STORE_F64 else torch.float32
        self._particles = None
        self._ckpt: list[torch.Tensor] = []
        self._win = None
        self._geo = None

    # ------------------------------------------------------------------
    def _setup(self, parr: np.ndarray) -> None:
        shape = (self.n,) * 3
        self._geo = DeviceGeometry(shape, self.subsamples, self.device, want_level=False, smooth_eps=self.eps)
        self._geo.set_particles(parr)
        self._geo.rebuild()
        self._win = LatticeWindow(shape, self.tau, self.force, self.subsamples, self.store, None, self.device)
        self._win.bind_geometry(self._geo)

    def forward(self, particles) -> float:
        """Run the window from rest for ``steps`` steps; return K (lattice units)."""
        parr = particles_array(particles)
        self._particles = parr
        with torch.cuda.device(self.device):
            self._setup(parr)
            win = self._win
            self._ckpt = []
            for t in range(self.steps):
                if t % self.every == 0:
                    self._ckpt.append(win.f[win.cur].clone())
                win.step(0)
            red = torch.zeros(nat.NRED, dtype=torch.float64, device=self.device)
            win.moments_pass(red, write_fields=False)
            r = red.cpu().numpy()
        flux = sum(self.dir[a] * r[nat.RED_FLUID_UX + a] for a in range(3))
        self.K = self.nu * flux / self.N / self.fmag
        return float(self.K)

    def _segment_states(self, t0: int, t1: int) -> torch.Tensor:
        """States S_t0 .. S_{t1-1} recomputed from the checkpoint at t0, shape (t1 - t0, 19 N)."""
        win = self._win
        L = t1 - t0
        buf = torch.empty((L, Q * self.N), dtype=self._fdtype, device=self.device)
        buf[0].copy_(self._ckpt[t0 // self.every])
        if L > 1:
            arr = (nat.PscWindow * (L - 1))()
            for k in range(L - 1):
                w = win.struct(0)
                w.f_src = buf[k].data_ptr()
                w.f_dst = buf[k + 1].data_ptr()
                w.imb = None
                w.moments = None
                arr[k] = w
            total = ctypes.c_int64(0)
            nat.call("psc_plan_tiles", arr, L - 1, 0, ctypes.byref(total))
            per = int(arr[0].tile_count)
            for k in range(L - 1):
                arr[k].tile_begin = 0
            table = struct_to_device(arr, self.device)
            size = ctypes.sizeof(nat.PscWindow)
            for k in range(L - 1):
                nat.call("psc_step_windows", self.store, ctypes.c_void_p(table.data_ptr() + k * size), 1, per,
                         nat.STEP_COLLIDE, 0, stream_handle(self.device))
        return buf

    def backward(self) -> np.ndarray:
        """dK/d(x, y, z, r) per particle, (P, 4), for the last forward()."""
        if self._win is None:
            raise RuntimeError("call forward() first")
        win, geo = self._win, self._geo
        N = self.N
        with torch.cuda.device(self.device):
            lam = [torch.empty(Q * N, dtype=self._fdtype, device=self.device) for _ in range(2)]
            dKdB = torch.zeros(N, dtype=torch.float64, device=self.device)
            dKds = torch.zeros(N, dtype=torch.float64, device=self.device)
            a = nat.PscAdjointArgs()
            a.nx = a.ny = a.nz = self.n
            a.store = self.store
            a.tau = self.tau
            a.force[0], a.force[1], a.force[2] = self.force
            a.kappa = self.kappa
            a.dir[0], a.dir[1], a.dir[2] = self.dir
            a.solid = vp(geo.solid)
            a.dKdB = vp(dKdB)
            a.dKdsolid = vp(dKds)
            a.state = vp(win.f[win.cur])
            a.lam_out = vp(lam[0])
            s = stream_handle(self.device)
            nat.call("psc_adjoint_seed", ctypes.byref(a), s)
            cur = 0
            nseg = (self.steps + self.every - 1) // self.every
            for seg in range(nseg - 1, -1, -1):
                t0 = seg * self.every
                t1 = min(t0 + self.every, self.steps)
                states = self._segment_states(t0, t1)
                for t in range(t1 - 1, t0 - 1, -1):
                    a.state = vp(states[t - t0])
                    a.lam_in = vp(lam[cur])
                    a.lam_out = vp(lam[1 - cur])
                    nat.call("psc_adjoint_step", ctypes.byref(a), s)
                    cur = 1 - cur
                del states
            P = geo.P
            grad = torch.zeros((max(P, 1), 4), dtype=torch.float64, device=self.device)
            g = geo.struct()
            part = geo.chunk_partials
            if part.numel() < geo.cap_chunks * 4:
                part = torch.zeros(geo.cap_chunks * 4, dtype=torch.float64, device=self.device)
            nat.call("psc_adjoint_geometry_grad", ctypes.byref(g), ctypes.byref(a), vp(part), vp(grad), s)
            self.dKdB = dKdB
            return grad[:P].cpu().numpy()

    def solid_gap(self) -> dict:
        """How far the smooth solid fraction is from the reference's counted one (same particles)."""
        if self._particles is None:
            raise RuntimeError("call forward() first")
        shape = (self.n,) * 3
        with torch.cuda.device(self.device):
            g = DeviceGeometry(shape, self.subsamples, self.device, want_level=False)
            g.set_particles(self._particles)
            g.rebuild()
            counted = g.solid
            diff = (self._geo.solid - counted).abs()
            return {"max_abs": float(diff.max().item()), "mean_abs": float(diff.mean().item()),
                    "solid_volume_smooth": float(self._geo.solid.sum().item()),
                    "solid_volume_counted": float(counted.sum().item())}


class _PermeabilityFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, centres: torch.Tensor, radii: torch.Tensor, problem: PermeabilityProblem, template):
        parts = np.array(template, dtype=np.float64, copy=True)
        parts[:, 0:3] = centres.detach().cpu().double().numpy()
        parts[:, 3] = radii.detach().cpu().double().numpy()
        K = problem.forward(parts)
        ctx.problem = problem
        return torch.tensor(K, dtype=torch.float64, device=centres.device)

    @staticmethod
    def backward(ctx, grad_out):
        g = torch.from_numpy(ctx.problem.backward()).to(device=grad_out.device)
        return grad_out * g[:, 0:3], grad_out * g[:, 3], None, None


def permeability(centres: torch.Tensor, radii: torch.Tensor, problem: PermeabilityProblem,
                 template: np.ndarray | None = None) -> torch.Tensor:
    """Darcy K as a differentiable function of particle centres (P, 3) and radii (P,)."""
    P = centres.shape[0]
    if template is None:
        template = np.zeros((P, 10))
    return _PermeabilityFn.apply(centres, radii, problem, template)
