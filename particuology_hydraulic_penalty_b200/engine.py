"""Device-side state of lattice windows and particle geometry.

PyTorch only allocates device memory and supplies the stream; every
computation is a call into libpscb200.so (``_native``).  There is no CPU
path: constructing anything here without a CUDA device raises.
"""

from __future__ import annotations

import ctypes
import operator
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as nat

PRECISIONS = {
    "fp64-exact": nat.STORE_F64_EXACT,
    "fp64": nat.STORE_F64,
    "fp32": nat.STORE_F32,
    "fp16": nat.STORE_F16,
    "bf16": nat.STORE_BF16,
}
STORE_DTYPE = {
    nat.STORE_F64_EXACT: torch.float64,
    nat.STORE_F64: torch.float64,
    nat.STORE_F32: torch.float32,
    nat.STORE_F16: torch.float16,
    nat.STORE_BF16: torch.bfloat16,
}
# element type of moments / imb / solid-velocity fields
FIELD_DTYPE = {
    nat.STORE_F64_EXACT: torch.float64,
    nat.STORE_F64: torch.float64,
    nat.STORE_F32: torch.float32,
    nat.STORE_F16: torch.float32,
    nat.STORE_BF16: torch.float32,
}
# FP16 stores deviation * 2^20: deviations of low-Mach flows (1e-8 .. 6e-2)
# land in FP16's normal range.  BF16 has FP32's exponent range.
DEFAULT_STORE_SCALE = {
    nat.STORE_F64_EXACT: 1.0,
    nat.STORE_F64: 1.0,
    nat.STORE_F32: 1.0,
    nat.STORE_F16: 2.0 ** 20,
    nat.STORE_BF16: 1.0,
}
Q = 19
PARTICLE_FIELDS = ("x", "y", "z", "r", "vx", "vy", "vz", "wx", "wy", "wz")
_particle_row = operator.attrgetter(*PARTICLE_FIELDS)


def trt_tau_minus(tau: float, magic: float = 3.0 / 16.0) -> float:
    """Antisymmetric relaxation time of TRT from the magic parameter
    Lambda = (tau - 1/2)(tau_minus - 1/2) (3/16 places bounce-back walls half-way)."""
    return 0.5 + magic / (tau - 0.5)


def check_inlet(inlet):
    """Normalise an inlet specification ``(rho_in, (ux, uy, uz))`` (None: periodic along x)."""
    if inlet is None:
        return None
    rho, u = inlet
    rho = float(rho)
    u = tuple(float(v) for v in u)
    if len(u) != 3 or not np.isfinite(rho) or rho <= 0.0 or not np.all(np.isfinite(u)):
        raise ValueError("inlet must be (rho_in > 0, (ux, uy, uz)) with finite values")
    return rho, u


def store_mode(precision: str) -> int:
    try:
        return PRECISIONS[precision]
    except KeyError:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {precision!r}") from None


def require_cuda(device=None) -> torch.device:
    """The CUDA device to use; raise when there is none (no CPU fallback)."""
    if not torch.cuda.is_available():
        raise RuntimeError("particuology_hydraulic_penalty_b200 runs on a CUDA GPU (B200, sm_100a) only; "
                           "no CUDA device is visible in this process")
    nat.load()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if dev.type != "cuda":
        raise ValueError(f"device must be a CUDA device, got {dev}")
    return dev


def vp(t: torch.Tensor | None):
    """Raw device pointer of a tensor (None for absent / empty)."""
    if t is None or t.numel() == 0:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_handle(device: torch.device | None = None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def particles_array(particles) -> np.ndarray:
    """(P, 10) float64 [x, y, z, r, vx, vy, vz, wx, wy, wz] from Particle3D-like objects or an array.

    Non-finite values raise ``ValueError`` (the reference fails on them when it
    converts the bounding box to integers, psc3d.py:73-78).
    """
    if isinstance(particles, np.ndarray):
        arr = np.ascontiguousarray(particles, dtype=np.float64)
        if arr.ndim != 2 or arr.shape[1] != 10:
            raise ValueError("a particle array must have shape (P, 10)")
    elif isinstance(particles, torch.Tensor):
        arr = np.ascontiguousarray(particles.detach().cpu().numpy(), dtype=np.float64)
        if arr.ndim != 2 or arr.shape[1] != 10:
            raise ValueError("a particle array must have shape (P, 10)")
    else:
        # one attribute tuple per particle (callers mutate Particle3D fields in place between steps)
        arr = np.array(list(map(_particle_row, particles)), dtype=np.float64).reshape(-1, 10)
    if not np.all(np.isfinite(arr)):
        raise ValueError("particle state contains NaN or Inf")
    return arr


def struct_to_device(structs, device) -> torch.Tensor:
    raw = bytes(memoryview(structs).cast("B"))
    host = torch.frombuffer(bytearray(raw), dtype=torch.uint8)
    return host.to(device, non_blocking=False)


# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------
class DeviceGeometry:
    """Particle-derived geometry of one window (wraps ``psc_geometry``).

    Holds the clipped boxes, per-entry inside counts, per-cell particle lists,
    ``alpha_sum``, ``solid`` and (for the non-exact storage modes) the uint8
    clipped sample level.  Buffers grow on demand; sizing needs one
    device-to-host read of the entry total per rebuild.
    """

    CHUNK_ENTRIES = 4096

    def __init__(self, shape, subsamples: int, device, want_level: bool, smooth_eps: float = 0.0):
        self.smooth_eps = float(smooth_eps)
        if self.smooth_eps < 0.0:
            raise ValueError("smooth_eps must be >= 0")
        if self.smooth_eps > 0.0:
            want_level = False  # a smooth solid fraction has no integer level
        self.nx, self.ny, self.nz = (int(v) for v in shape)
        self.subsamples = int(subsamples)
        if self.subsamples < 1 or self.subsamples > 16:
            raise ValueError("subsamples must be in [1, 16]")
        if want_level and self.subsamples ** 3 > 255:
            raise ValueError("the FP32/FP16/BF16 and fast-FP64 modes store the solid level as uint8 "
                             "and need subsamples <= 6")
        self.device = device
        self.N = self.nx * self.ny * self.nz
        N = self.N
        i32, i64, f64 = torch.int32, torch.int64, torch.float64
        self.cell_n = torch.zeros(N, dtype=i32, device=device)
        self.cell_off = torch.zeros(N + 1, dtype=i32, device=device)
        self.alpha_sum = torch.zeros(N, dtype=f64, device=device)
        self.solid = torch.zeros(N, dtype=f64, device=device)
        self.level = torch.zeros(N, dtype=torch.uint8, device=device) if want_level else None
        self.scan_tmp = torch.zeros(int(nat.load().psc_scan_tmp_bytes(N + 1)), dtype=torch.uint8, device=device)
        self.totals = torch.zeros(4, dtype=i64, device=device)
        self.P = -1
        self.particles = torch.zeros((0, 10), dtype=f64, device=device)
        self._pinned = None
        self._upload_done = None
        self.bbox = self.ent_off = self.chunk_off = None
        self.cap_entries = 0
        self.cap_chunks = 0
        self.ent_cnt = torch.zeros(0, dtype=torch.int16, device=device)
        self.cl_pid = torch.zeros(0, dtype=i32, device=device)
        self.cl_cnt = torch.zeros(0, dtype=torch.int16, device=device)
        self.ent_alpha = None
        self.cl_ent = None
        self.chunk_partials = torch.zeros(0, dtype=f64, device=device)
        self.n_entries = 0
        self.n_chunks = 0
        self.built = False
        self.host_particles = np.zeros((0, 10))

    def set_particles(self, arr: np.ndarray) -> bool:
        """Upload the (P, 10) particle state (positions, radii, velocities, spins).

        Staged through a pinned host buffer and copied asynchronously on the
        current stream (every call: callers may mutate particles in place).
        Returns True when the state differs from the previous upload.
        """
        P = arr.shape[0]
        if P != self.P:
            dev = self.device
            self.P = P
            self.bbox = torch.zeros(max(P, 1) * 6, dtype=torch.int32, device=dev)
            self.ent_off = torch.zeros(P + 1, dtype=torch.int64, device=dev)
            self.chunk_off = torch.zeros(P + 1, dtype=torch.int64, device=dev)
            self.particles = torch.zeros((P, 10), dtype=torch.float64, device=dev)
            self._pinned = torch.zeros((max(P, 1), 10), dtype=torch.float64).pin_memory()
            self._upload_done = None
            self.built = False
            self.host_particles = np.zeros((0, 10))
        changed = not (self.host_particles.shape == arr.shape and np.array_equal(self.host_particles, arr))
        self.host_particles = arr.copy()
        if P:
            if self._upload_done is not None:
                self._upload_done.synchronize()  # the pinned buffer is free again
            self._pinned[:P].numpy()[...] = arr
            self.particles.copy_(self._pinned[:P], non_blocking=True)
            self._upload_done = torch.cuda.Event()
            self._upload_done.record()
        return changed

    def struct(self) -> nat.PscGeometry:
        """The psc_geometry descriptor (cached; rebuilt when a buffer or size changes)."""
        key = (self.P, self.cap_entries, self.cap_chunks, self.particles.data_ptr() if self.particles.numel() else 0,
               self.bbox.data_ptr() if self.bbox is not None else 0)
        if getattr(self, "_struct_key", None) != key:
            self._struct_cache = self._make_struct()
            self._struct_key = key
        return nat.PscGeometry.from_buffer_copy(self._struct_cache)  # callers may edit their copy

    def _make_struct(self) -> nat.PscGeometry:
        g = nat.PscGeometry()
        g.nx, g.ny, g.nz = self.nx, self.ny, self.nz
        g.subsamples = self.subsamples
        g.nparticles = self.P
        g.chunk_entries = self.CHUNK_ENTRIES
        g.capacity_entries = self.cap_entries
        g.capacity_chunks = self.cap_chunks
        g.particles = vp(self.particles)
        g.bbox = vp(self.bbox)
        g.ent_off = vp(self.ent_off)
        g.chunk_off = vp(self.chunk_off)
        g.totals = vp(self.totals)
        g.ent_cnt = vp(self.ent_cnt)
        g.cell_n = vp(self.cell_n)
        g.cell_off = vp(self.cell_off)
        g.cl_pid = vp(self.cl_pid)
        g.cl_cnt = vp(self.cl_cnt)
        g.alpha_sum = vp(self.alpha_sum)
        g.solid = vp(self.solid)
        g.level = vp(self.level)
        g.scan_tmp = vp(self.scan_tmp)
        g.smooth_eps = self.smooth_eps
        g.ent_alpha = vp(self.ent_alpha)
        g.cl_ent = vp(self.cl_ent)
        return g

    def rebuild(self) -> None:
        """Voxelise the current particles (psc3d.py:151-179 / 328-345)."""
        if self.P < 0:
            raise RuntimeError("set_particles() before rebuild()")
        s = stream_handle(self.device)
        g = self.struct()
        nat.call("psc_geometry_plan", ctypes.byref(g), s)
        tot = self.totals.cpu().numpy()
        self.n_entries, self.n_chunks = int(tot[0]), int(tot[1])
        if self.n_entries >= 2 ** 31 - 1:
            raise ValueError("too many bounding-box entries (>= 2^31) for one window")
        if self.n_entries > self.cap_entries:
            cap = int(self.n_entries * 1.25) + 1024
            cap = min(cap, 2 ** 31 - 2)
            self.ent_cnt = torch.zeros(cap, dtype=torch.int16, device=self.device)
            self.cl_pid = torch.zeros(cap, dtype=torch.int32, device=self.device)
            self.cl_cnt = torch.zeros(cap, dtype=torch.int16, device=self.device)
            if self.smooth_eps > 0.0:
                self.ent_alpha = torch.zeros(cap, dtype=torch.float64, device=self.device)
                self.cl_ent = torch.zeros(cap, dtype=torch.int32, device=self.device)
            self.cap_entries = cap
        if self.n_chunks > self.cap_chunks:
            cap = int(self.n_chunks * 1.25) + 16
            self.chunk_partials = torch.zeros(cap * 6, dtype=torch.float64, device=self.device)
            self.cap_chunks = cap
        g = self.struct()
        nat.call("psc_geometry_build", ctypes.byref(g), s)
        self.built = True

    def solid_velocity(self, out: torch.Tensor) -> None:
        g = self.struct()
        us_type = 0 if out.dtype == torch.float64 else 1
        nat.call("psc_solid_velocity", ctypes.byref(g), us_type, vp(out), stream_handle(self.device))

    def loads(self, imb: torch.Tensor, imb_sums: torch.Tensor, forces: torch.Tensor, torques: torch.Tensor,
              diag: torch.Tensor) -> None:
        g = self.struct()
        imb_type = 0 if imb.dtype == torch.float64 else 1
        nat.call("psc_particle_loads", ctypes.byref(g), imb_type, vp(imb), vp(self.chunk_partials), vp(imb_sums),
                 vp(forces), vp(torques), vp(diag), stream_handle(self.device))

    # -- host views used by the drop-in classes (tests / small lattices) --
    def sparse_lists(self):
        """Per-particle ascending node ids and alphas, like SparsePscD3Q19.node_ids / alpha_vals."""
        P = max(self.P, 0)
        if P == 0:
            return [], []
        cnt = self.ent_cnt[: self.n_entries].cpu().numpy().astype(np.int64)
        off = self.ent_off.cpu().numpy()
        bbox = self.bbox.cpu().numpy().reshape(-1, 6)
        s3 = float(self.subsamples ** 3)
        ids_l, vals_l = [], []
        for p in range(P):
            x0, y0, z0, ex, ey, ez = (int(v) for v in bbox[p])
            c = cnt[off[p]: off[p + 1]]
            if c.size == 0:
                ids_l.append(np.zeros(0, dtype=np.int64))
                vals_l.append(np.zeros(0))
                continue
            loc = np.nonzero(c)[0]
            a = loc // (ey * ez)
            rem = loc - a * ey * ez
            b = rem // ez
            k = rem - b * ez
            ids = ((a + x0) * self.ny + (b + y0)) * self.nz + (k + z0)
            ids_l.append(ids.astype(np.int64))
            vals_l.append(c[loc] / s3)
        return ids_l, vals_l


# ---------------------------------------------------------------------------
# one lattice window
# ---------------------------------------------------------------------------
@dataclass
class StepResult:
    """Host copies produced by one reporting step."""

    red_pre: np.ndarray  # reductions of the pre-collision (pulled) state + this step's imb sums
    red_post: np.ndarray  # reductions of the post-stream state (after the step)
    diag: np.ndarray  # psc_particle_loads diagnostics


class LatticeWindow:
    """Populations and per-cell fields of one periodic window on the device."""

    def __init__(self, shape, tau: float, force, subsamples: int, store: int, store_scale: float | None,
                 device, tau_minus: float = 0.0, inlet=None):
        self.nx, self.ny, self.nz = (int(v) for v in shape)
        # inlet = (rho_in, (ux, uy, uz)): open along x (PSC_WIN_OPEN_X), else periodic
        self.inlet = check_inlet(inlet)
        self.N = self.nx * self.ny * self.nz
        self.tau = float(tau)
        self.tau_minus = float(tau_minus)
        self.force = tuple(float(v) for v in force)
        self.subsamples = int(subsamples)
        self.store = int(store)
        if self.tau_minus > 0.0 and self.store == nat.STORE_F64_EXACT:
            raise ValueError("TRT collision runs in the deviation storage modes (fp64, fp32, fp16, bf16)")
        self.store_scale = float(DEFAULT_STORE_SCALE[self.store] if store_scale is None else store_scale)
        if self.store_scale <= 0.0 or not np.isfinite(self.store_scale):
            raise ValueError("store_scale must be a positive finite number")
        self.device = device
        sd, fd = STORE_DTYPE[self.store], FIELD_DTYPE[self.store]
        N = self.N
        self.f = [torch.empty(Q * N, dtype=sd, device=device), torch.empty(Q * N, dtype=sd, device=device)]
        self.cur = 0
        self.imb: torch.Tensor | None = None  # [3][N], allocated on first use
        self.moments: torch.Tensor | None = None  # [4][N], allocated on first use
        self.us: torch.Tensor | None = None
        self.red = torch.zeros(nat.NRED, dtype=torch.float64, device=device)
        self.red_post = torch.zeros(nat.NRED, dtype=torch.float64, device=device)
        self.solid_ptr = None
        self.level_ptr = None
        self.moving = False
        nat.call("psc_init_equilibrium", self.store, self.store_scale, vp(self.f[0]), N, stream_handle(device))
        self.tiles = 0
        self.partials = None
        self._win_dev = [None, None]
        self._dirty = True

    # window descriptor ----------------------------------------------------
    def bind_geometry(self, geo: DeviceGeometry) -> None:
        self.solid_ptr = vp(geo.solid)
        self.level_ptr = vp(geo.level)
        self._dirty = True

    def ensure_fields(self, imb: bool = True, moments: bool = True) -> None:
        fd = FIELD_DTYPE[self.store]
        if imb and self.imb is None:
            self.imb = torch.zeros(3 * self.N, dtype=fd, device=self.device)
            self._dirty = True
        if moments and self.moments is None:
            self.moments = torch.zeros(4 * self.N, dtype=fd, device=self.device)
            self._dirty = True

    def ensure_us(self) -> torch.Tensor:
        if self.us is None:
            self.us = torch.zeros(3 * self.N, dtype=FIELD_DTYPE[self.store], device=self.device)
            self._dirty = True
        return self.us

    def set_moving(self, moving: bool) -> None:
        if moving != self.moving:
            self.moving = moving
            self._dirty = True

    def struct(self, src: int) -> nat.PscWindow:
        """The psc_window descriptor reading buffer ``src`` (tile fields unset)."""
        return self._struct(src)

    def _struct(self, src: int) -> nat.PscWindow:
        w = nat.PscWindow()
        w.nx, w.ny, w.nz = self.nx, self.ny, self.nz
        w.subsamples = self.subsamples
        w.flags = (nat.WIN_MOVING if self.moving else 0) | (nat.WIN_OPEN_X if self.inlet else 0)
        w.tau = self.tau
        w.tau_minus = self.tau_minus
        if self.inlet:
            w.inlet_rho = self.inlet[0]
            w.inlet_u[0], w.inlet_u[1], w.inlet_u[2] = self.inlet[1]
        else:
            w.inlet_rho = 1.0
        w.force[0], w.force[1], w.force[2] = self.force
        w.store_scale = self.store_scale
        w.f_src = vp(self.f[src])
        w.f_dst = vp(self.f[1 - src])
        w.solid = self.solid_ptr
        w.level = self.level_ptr
        w.us = vp(self.us) if self.moving else None
        w.imb = vp(self.imb)
        w.moments = vp(self.moments)
        return w

    def windows(self, src: int) -> torch.Tensor:
        if self._dirty:
            structs = []
            for s in (0, 1):
                w = self._struct(s)
                total = ctypes.c_int64(0)
                nat.call("psc_plan_tiles", ctypes.byref(w), 1, 0, ctypes.byref(total))
                if self.partials is None or self.tiles != total.value:
                    self.tiles = total.value
                    self.partials = torch.zeros((1 + self.tiles * nat.PARTIAL_ROWS) * nat.NRED, dtype=torch.float64,
                                                device=self.device)
                w.partials = vp(self.partials)
                structs.append(w)
            self._win_dev = [struct_to_device(structs[0], self.device), struct_to_device(structs[1], self.device)]
            self._dirty = False
        return self._win_dev[src]

    # kernels ----------------------------------------------------------------
    def step(self, flags: int) -> None:
        """One fused pull-stream + collide step; swaps the population buffers."""
        self.ensure_fields(imb=bool(flags & nat.STEP_IMB), moments=bool(flags & nat.STEP_MOMENTS))
        if self.solid_ptr is None:
            raise RuntimeError("geometry not bound")
        fl = flags | nat.STEP_COLLIDE | (nat.STEP_MOVING if self.moving else 0)
        nat.call("psc_step_windows", self.store, vp(self.windows(self.cur)), 1, self.tiles, fl, 0,
                 stream_handle(self.device))
        self.cur = 1 - self.cur

    def reduce(self, out: torch.Tensor) -> None:
        nat.call("psc_reduce_windows", vp(self.windows(self.cur)), 1, vp(out), stream_handle(self.device))

    def moments_pass(self, reduce_out: torch.Tensor | None = None, write_fields: bool = True) -> None:
        """Moments (and reductions) of the current post-stream state, no collision."""
        self.ensure_fields(imb=False, moments=write_fields)
        fl = (nat.STEP_MOMENTS if write_fields else 0) | (nat.STEP_REDUCE if reduce_out is not None else 0)
        nat.call("psc_step_windows", self.store, vp(self.windows(self.cur)), 1, self.tiles, fl, 0,
                 stream_handle(self.device))
        if reduce_out is not None:
            self.reduce(reduce_out)

    def post_stream_f(self) -> torch.Tensor:
        """Absolute FP64 post-stream populations (19, nx, ny, nz) on the device."""
        out = torch.empty(Q * self.N, dtype=torch.float64, device=self.device)
        if self.inlet:
            u = (ctypes.c_double * 3)(*self.inlet[1])
            nat.call("psc_stream_push_open", self.store, self.store_scale, vp(self.f[self.cur]), vp(out), self.nx,
                     self.ny, self.nz, self.inlet[0], u, stream_handle(self.device))
        else:
            nat.call("psc_stream_push", self.store, self.store_scale, vp(self.f[self.cur]), vp(out), self.nx, self.ny,
                     self.nz, stream_handle(self.device))
        return out.view(Q, self.nx, self.ny, self.nz)

    def load_post_stream_f(self, f: torch.Tensor) -> None:
        """Set the state from absolute FP64 post-stream populations (19, nx, ny, nz)."""
        src = f.to(device=self.device, dtype=torch.float64).contiguous().view(-1)
        if src.numel() != Q * self.N:
            raise ValueError(f"f must have {Q}x{self.nx}x{self.ny}x{self.nz} elements")
        if self.inlet:
            u = (ctypes.c_double * 3)(*self.inlet[1])
            nat.call("psc_stream_pull_store_open", self.store, self.store_scale, vp(src), vp(self.f[self.cur]),
                     self.nx, self.ny, self.nz, self.inlet[0], u, stream_handle(self.device))
        else:
            nat.call("psc_stream_pull_store", self.store, self.store_scale, vp(src), vp(self.f[self.cur]), self.nx,
                     self.ny, self.nz, stream_handle(self.device))
