"""Many pore windows of uneven size stepped by one persistent launch.

Every step is ONE ``psc_step_windows_ex`` launch whose persistent grid walks the tiles
of all windows; the windows' descriptors sit in two device tables (even and
odd step parity).  Step sequences are captured once in a CUDA graph and
replayed, so a run issues no per-step host work.  Reductions (Darcy flux,
porosity, NaN count) are taken only on reporting steps, in FP64, per window.

This is the throughput path for permeability campaigns (the reference runs
one NumPy solver per window and resolution,
scripts/run_psc_permeability_resolution.py:122-192); the drop-in classes in
``psc3d`` keep the reference's per-call semantics.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as nat
from .engine import (DeviceGeometry, LatticeWindow, particles_array, require_cuda, store_mode, stream_handle,
                     struct_to_device, trt_tau_minus, vp)


@dataclass
class WindowSpec:
    """One lattice window of a batch."""

    n: int
    particles: np.ndarray  # (P, 10)
    tau: float = 0.8
    force: tuple = (1.0e-6, 0.0, 0.0)
    subsamples: int = 4
    name: str = ""
    collision: str = "bgk"  # "bgk" (the reference) or "trt" (magic parameter 3/16)
    inlet: tuple | None = None  # (rho_in, (ux, uy, uz)): velocity inlet at x = 0, outflow at x = nx - 1


class PscBatch:
    """A batch of independent periodic windows advanced together.

    Parameters
    ----------
    specs : list of WindowSpec (or objects with ``n`` and ``particles``)
    precision : storage mode ("fp64-exact", "fp64", "fp32", "fp16", "bf16")
    graph_steps : steps per captured CUDA graph (0 disables graphs)
    grid_ctas : persistent grid size (0 = SM count x occupancy)
    """

    def __init__(self, specs, precision: str = "fp32", store_scale: float | None = None, graph_steps: int = 20,
                 grid_ctas: int = 0, device=None, tau=None, force=None, subsamples=None, cells_per_thread: int = 1,
                 kernel: int = nat.KERNEL_AUTO, tile_rows: int = 0, stages: int = 3):
        self.device = require_cuda(device)
        self.store = store_mode(precision)
        self.precision = precision
        self.cells_per_thread = 1 if self.store == nat.STORE_F64_EXACT else int(cells_per_thread)
        if self.cells_per_thread not in (1, 2, 4):
            raise ValueError("cells_per_thread must be 1, 2 or 4")
        self.kernel = int(kernel)
        if self.kernel in (nat.KERNEL_TMA, nat.KERNEL_PAIR) and self.store == nat.STORE_F64_EXACT:
            raise ValueError("the TMA and pair kernels run the deviation storage modes")
        self.tile_rows = int(tile_rows)
        self.rows_per_window: list[int] | None = None  # per-window TMA rows (autotuner), else tile_rows
        self.stages = int(stages)
        self.stage_bytes = 0
        self.graph_steps = int(graph_steps)
        if self.graph_steps % 2:
            raise ValueError("graph_steps must be even (the graph must end on the buffer parity it started on)")
        self.grid_ctas = int(grid_ctas)
        self.specs = []
        for s in specs:
            if not isinstance(s, WindowSpec):
                s = WindowSpec(n=int(s.n), particles=np.asarray(s.particles), name=getattr(s, "kind", ""))
            if tau is not None:
                s.tau = float(tau)
            if force is not None:
                s.force = tuple(float(v) for v in force)
            if subsamples is not None:
                s.subsamples = int(subsamples)
            self.specs.append(s)
        if not self.specs:
            raise ValueError("a batch needs at least one window")
        self.windows: list[LatticeWindow] = []
        self.geoms: list[DeviceGeometry] = []
        with torch.cuda.device(self.device):
            for s in self.specs:
                shape = (s.n, s.n, s.n)
                if s.collision not in ("bgk", "trt"):
                    raise ValueError("collision must be 'bgk' or 'trt'")
                tm = trt_tau_minus(s.tau) if s.collision == "trt" else 0.0
                win = LatticeWindow(shape, s.tau, s.force, s.subsamples, self.store, store_scale, self.device,
                                    tau_minus=tm, inlet=getattr(s, "inlet", None))
                geo = DeviceGeometry(shape, s.subsamples, self.device, want_level=self.store != nat.STORE_F64_EXACT)
                geo.set_particles(particles_array(s.particles))
                geo.rebuild()
                win.bind_geometry(geo)
                self.windows.append(win)
                self.geoms.append(geo)
        self.cells = np.array([w.N for w in self.windows], dtype=np.int64)
        self.parity = 0
        self.steps_done = 0
        self.frozen: dict[int, int] = {}  # window -> buffer parity holding its frozen state
        self._frozen_red: dict[int, np.ndarray] = {}
        self._tables = None
        self._graphs: dict = {}
        self._red = torch.zeros(len(self.windows) * nat.NRED, dtype=torch.float64, device=self.device)
        self._build_tables()

    # ------------------------------------------------------------------
    def _resolve_kernel(self) -> int:
        """KERNEL_AUTO: the pair kernel for FP32/FP16/BF16 storage when every window has an even nz and
        one cell per thread is asked for (measured +9 % on the 24-window batch), else the direct kernel
        (FP64 pairs need about 240 registers per thread: one CTA per SM)."""
        if self.kernel != nat.KERNEL_AUTO:
            return self.kernel
        if (self.store in (nat.STORE_F32, nat.STORE_F16, nat.STORE_BF16) and self.cells_per_thread == 1
                and all(w.nz % 2 == 0 for w in self.windows)):
            return nat.KERNEL_PAIR
        return nat.KERNEL_DIRECT

    def _build_tables(self) -> None:
        nwin = len(self.windows)
        tables = []
        self.partials = None
        self.kernel_eff = self._resolve_kernel()
        for parity in (0, 1):
            arr = (nat.PscWindow * nwin)()
            for k, w in enumerate(self.windows):
                arr[k] = w.struct(parity)
                if k in self.frozen:
                    arr[k].flags |= nat.WIN_INACTIVE
                if self.rows_per_window is not None:
                    arr[k].tile_cells = int(self.rows_per_window[k]) * w.nz
            total = ctypes.c_int64(0)
            if self.kernel_eff == nat.KERNEL_TMA:
                sb = ctypes.c_int32(0)
                elem = self.windows[0].f[0].element_size()
                rows = -1 if self.rows_per_window is not None else self.tile_rows
                nat.call("psc_plan_row_tiles", arr, nwin, rows, elem, ctypes.byref(total), ctypes.byref(sb))
                self.stage_bytes = int(sb.value)
            elif self.kernel_eff == nat.KERNEL_PAIR:
                nat.call("psc_plan_pair_tiles", arr, nwin, ctypes.byref(total))
            else:
                nat.call("psc_plan_tiles", arr, nwin, nat.STEP_THREADS * self.cells_per_thread, ctypes.byref(total))
            if self.partials is None:
                self.total_tiles = int(total.value)
                # per window: a header row, then up to tile_count * PARTIAL_ROWS rows
                self.partials = torch.zeros((nwin + self.total_tiles * nat.PARTIAL_ROWS) * nat.NRED,
                                            dtype=torch.float64, device=self.device)
            base = self.partials.data_ptr()
            for k in range(nwin):
                arr[k].partials = base + (k + int(arr[k].tile_begin) * nat.PARTIAL_ROWS) * nat.NRED * 8
            tables.append(struct_to_device(arr, self.device))
        self._tables = tables
        self._graphs = {}

    def configure(self, kernel: int, cells_per_thread: int = 1, tile_rows: int = 0, stages: int = 3,
                  rows_per_window=None, grid_ctas: int | None = None) -> None:
        """Switch the launch configuration (populations are kept; graphs are re-captured)."""
        if kernel in (nat.KERNEL_TMA, nat.KERNEL_PAIR) and self.store == nat.STORE_F64_EXACT:
            raise ValueError("the TMA and pair kernels run the deviation storage modes")
        self.kernel = int(kernel)
        self.cells_per_thread = int(cells_per_thread)
        self.tile_rows = int(tile_rows)
        self.stages = int(stages)
        self.rows_per_window = None if rows_per_window is None else [int(r) for r in rows_per_window]
        if grid_ctas is not None:
            self.grid_ctas = int(grid_ctas)
        self._build_tables()

    def launch_config(self) -> dict:
        return {"kernel": {nat.KERNEL_DIRECT: "direct", nat.KERNEL_TMA: "tma",
                           nat.KERNEL_PAIR: "pair"}[self.kernel_eff],
                "cells_per_thread": self.cells_per_thread, "tile_rows": self.tile_rows, "stages": self.stages,
                "rows_per_window": self.rows_per_window, "stage_bytes": self.stage_bytes,
                "grid_ctas": self.grid_ctas}

    @property
    def nwin(self) -> int:
        return len(self.windows)

    @property
    def total_cells(self) -> int:
        return int(self.cells.sum())

    def _launch(self, flags: int) -> None:
        cfg = nat.PscLaunch(self.grid_ctas, self.cells_per_thread, self.kernel_eff, self.stages, self.stage_bytes)
        nat.call("psc_step_windows_ex", self.store, vp(self._tables[self.parity]), self.nwin, self.total_tiles,
                 flags, ctypes.byref(cfg), stream_handle(self.device))

    def _sync_cur(self) -> None:
        for k, w in enumerate(self.windows):
            w.cur = self.frozen.get(k, self.parity)

    def step_once(self, flags: int = 0) -> None:
        """One collide-stream step of every active window (one kernel launch)."""
        self._launch(flags | nat.STEP_COLLIDE)
        self.parity ^= 1
        self._sync_cur()
        self.steps_done += 1

    def freeze(self, k: int, red_row: np.ndarray | None = None) -> None:
        """Stop stepping window k (its tiles are skipped by the kernel); keeps its current state.

        The flag is written into both device tables in place, so captured step
        graphs stay valid.
        """
        if k in self.frozen:
            return
        self.frozen[k] = self.parity
        if red_row is not None:
            self._frozen_red[k] = np.array(red_row, dtype=np.float64)
        size = ctypes.sizeof(nat.PscWindow)
        off = nat.PscWindow.flags.offset
        for table in self._tables:
            cur = int(table[k * size + off: k * size + off + 4].view(torch.int32).item())
            table[k * size + off: k * size + off + 4].copy_(
                torch.tensor([cur | nat.WIN_INACTIVE], dtype=torch.int32).view(torch.uint8))
        self._sync_cur()

    def _capture(self) -> None:
        """Capture graph_steps launches starting at the current buffer parity."""
        g = torch.cuda.CUDAGraph()
        stream = torch.cuda.Stream(self.device)
        stream.wait_stream(torch.cuda.current_stream(self.device))
        parity0 = self.parity
        with torch.cuda.stream(stream):
            with torch.cuda.graph(g, stream=stream):
                for _ in range(self.graph_steps):
                    self._launch(nat.STEP_COLLIDE)
                    self.parity ^= 1
        torch.cuda.current_stream(self.device).wait_stream(stream)
        self.parity = parity0
        self._graphs[parity0] = g

    def prepare(self) -> None:
        """Warm the launch path and capture the step graphs of both buffer parities (no timed work)."""
        with torch.cuda.device(self.device):
            if self.steps_done == 0:
                self.step_once()
            if self.graph_steps > 0:
                for _ in range(2):
                    if self.parity not in self._graphs:
                        self._capture()
                    self.parity ^= 1  # capture does not run anything; visit the other parity
                self._sync_cur()

    def run(self, steps: int) -> None:
        """Advance every window by ``steps`` steps (graph replays plus a remainder)."""
        steps = int(steps)
        with torch.cuda.device(self.device):
            if self.graph_steps > 0 and steps >= self.graph_steps:
                if self.steps_done == 0 or len(self._graphs) < 2:
                    steps -= 1 if self.steps_done == 0 else 0
                    self.prepare()
                graph = self._graphs[self.parity]  # an even step count returns to this parity
                reps = steps // self.graph_steps
                for _ in range(reps):
                    graph.replay()
                self.steps_done += reps * self.graph_steps
                steps -= reps * self.graph_steps
                self._sync_cur()
            for _ in range(steps):
                self.step_once()

    def launches_per_step(self) -> int:
        return 1

    # ------------------------------------------------------------------
    def observe(self) -> np.ndarray:
        """FP64 reductions of every window's current post-stream state, (nwin, NRED) on the host."""
        with torch.cuda.device(self.device):
            self._launch(nat.STEP_REDUCE)
            nat.call("psc_reduce_windows", vp(self._tables[self.parity]), self.nwin, vp(self._red),
                     stream_handle(self.device))
            red = self._red.view(self.nwin, nat.NRED).cpu().numpy().copy()
        for k, row in self._frozen_red.items():  # frozen windows wrote no partials
            red[k] = row
        return red

    def permeability(self, red: np.ndarray | None = None) -> np.ndarray:
        """Darcy K per window along its body force, run_psc_permeability_resolution.py:144-150."""
        red = self.observe() if red is None else red
        out = np.zeros(self.nwin)
        for k, s in enumerate(self.specs):
            F = np.asarray(s.force, dtype=float)
            fmag = float(np.linalg.norm(F))
            d = F / max(fmag, 1e-300)
            flux = d[0] * red[k, nat.RED_FLUID_UX] + d[1] * red[k, nat.RED_FLUID_UY] + d[2] * red[k, nat.RED_FLUID_UZ]
            superficial = flux / float(self.cells[k])
            nu = (s.tau - 0.5) / 3.0
            out[k] = nu * superficial / max(fmag, 1e-300)
        return out

    def run_to_convergence(self, tol: float = 1.0e-8, check_every: int = 200, max_steps: int = 200000,
                           min_steps: int = 0, freeze: bool = True) -> dict:
        """Step until every window's per-step relative change of K is below ``tol``.

        The criterion of the reference's coupled driver, |q_k - q_{k-1}| / |q_k| <
        tol between consecutive steps (coupling_sync/couple_psc_liggghts.py:284-296),
        applied to the Darcy flux of each window and evaluated on a pair of
        consecutive steps every ``check_every`` steps (no per-step host work in
        between).  A window that converges is frozen (``freeze``): the kernel skips
        its tiles from then on, so the launch spends HBM bandwidth only on the
        windows still converging.  Returns per-window steps, residuals and K.
        """
        nwin = self.nwin
        conv_step = np.full(nwin, -1, dtype=np.int64)
        residual = np.full(nwin, np.inf)
        start = self.steps_done
        while True:
            done = self.steps_done - start
            if done >= max_steps:
                break
            self.run(max(0, min(check_every - 1, max_steps - done - 1)))
            k1 = self.permeability()
            self.run(1)
            red = self.observe()
            k2 = self.permeability(red)
            if self.nonfinite(red).any():
                raise FloatingPointError("non-finite moments in window(s) "
                                         f"{np.nonzero(self.nonfinite(red))[0].tolist()}")
            residual = np.abs(k2 - k1) / np.maximum(np.abs(k2), 1e-300)
            now = self.steps_done - start
            newly = (conv_step < 0) & (residual < tol) & (now >= min_steps)
            conv_step[newly] = now
            if freeze:
                for k in np.nonzero(newly)[0]:
                    self.freeze(int(k), red[k])
            if np.all(conv_step >= 0):
                break
        return {"steps": conv_step, "residual": residual, "permeability": self.permeability(),
                "converged": conv_step >= 0, "total_steps": self.steps_done - start}

    def nonfinite(self, red: np.ndarray | None = None) -> np.ndarray:
        red = self.observe() if red is None else red
        return red[:, nat.RED_NONFINITE] > 0

    def loads(self) -> list[tuple[np.ndarray, np.ndarray]]:
        """Per-particle force and torque of every window from one extra collide step."""
        out = []
        with torch.cuda.device(self.device):
            self._ensure_imb()
            self.step_once(nat.STEP_IMB | nat.STEP_REDUCE)
            nat.call("psc_reduce_windows", vp(self._tables[self.parity]), self.nwin, vp(self._red),
                     stream_handle(self.device))
            for k, (w, g) in enumerate(zip(self.windows, self.geoms)):
                P = g.P
                F = torch.zeros((P, 3), dtype=torch.float64, device=self.device)
                T = torch.zeros((P, 3), dtype=torch.float64, device=self.device)
                diag = torch.zeros(nat.NDIAG, dtype=torch.float64, device=self.device)
                g.loads(w.imb, self._red[k * nat.NRED + nat.RED_IMBX:], F, T, diag)
                out.append((F.cpu().numpy(), T.cpu().numpy()))
        return out

    def _ensure_imb(self) -> None:
        if any(w.imb is None for w in self.windows):
            for w in self.windows:
                w.ensure_fields(imb=True, moments=False)
            self._build_tables()

    def velocity_field(self, k: int) -> np.ndarray:
        """(4, n, n, n) rho, ux, uy, uz of window k's post-stream state (FP64 host copy)."""
        w = self.windows[k]
        with torch.cuda.device(self.device):
            w.cur = self.parity
            w.moments_pass(None, write_fields=True)
            return w.moments.to(torch.float64).view(4, w.nx, w.ny, w.nz).cpu().numpy()
