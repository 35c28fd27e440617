"""Project-written autotuner for the batched step launch.

Candidates (all compute identical per-cell arithmetic, so the choice only
changes speed):
  * direct kernel, 1 or 2 cells per thread;
  * pair kernel (two consecutive z cells per thread, 2-element accesses),
    when every window has an even nz;
  * for the direct (1 cell per thread) and pair kernels, the persistent grid:
    the occupancy default, or 1, 2 or 4 CTAs per SM (each CTA walks a
    contiguous run of tiles; more CTAs than fit run in waves);
  * TMA row-staged kernel, 2 / 3 / 4 pipeline stages, with the rows per tile
    chosen per window SIZE CLASS (windows of equal extent share a class).

Procedure: for each size class, time the TMA row candidates on that class
alone (CUDA events, a few steps after warm-up); then time the full batch once
per kernel / stage candidate with each class at its best rows; keep the
fastest.  The populations are snapshotted before and restored after, so
tuning does not advance the simulation.  Results are cached per GPU name,
storage mode and window-class multiset in a JSON file
($PSC_B200_CACHE or ~/.cache/psc_b200/autotune.json).
"""

from __future__ import annotations

import json
import os
from pathlib import Path

import torch

from . import _native as nat

CACHE_ENV = "PSC_B200_CACHE"


def cache_path() -> Path:
    p = os.environ.get(CACHE_ENV)
    return Path(p) if p else Path.home() / ".cache" / "psc_b200" / "autotune.json"


def _key(batch) -> str:
    name = torch.cuda.get_device_name(batch.device)
    classes = sorted({(w.nx, w.ny, w.nz) for w in batch.windows})
    counts = {c: sum(1 for w in batch.windows if (w.nx, w.ny, w.nz) == c) for c in classes}
    return json.dumps([name, batch.precision, [[list(c), counts[c]] for c in classes]])


def _time(batch, steps: int, warm: int = 3) -> float:
    batch.run(warm)
    torch.cuda.synchronize(batch.device)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    batch.run(steps)
    b.record()
    torch.cuda.synchronize(batch.device)
    return a.elapsed_time(b) / steps


def _snapshot(batch):
    return [w.f[batch.parity].clone() for w in batch.windows], batch.parity, batch.steps_done


def _restore(batch, snap):
    states, parity, steps_done = snap
    for w, s in zip(batch.windows, states):
        w.f[parity].copy_(s)
        w.cur = parity
    batch.parity = parity
    batch.steps_done = steps_done


def _row_candidates(nz: int, ny: int, elem: int, stages: int = 2) -> list[int]:
    per_row = nz * (19 * elem + 1)
    auto = max(1, (24 * 1024) // per_row)
    cands = {1, 2, 4, 8, auto, max(1, auto // 2), auto * 2, auto * 4}
    return sorted(r for r in cands
                  if r <= ny and r * per_row <= 96 * 1024 and r * per_row * stages <= 200 * 1024 and r * nz <= 4096)


def tune(batch, steps: int = 20, use_cache: bool = True, verbose: bool = False) -> dict:
    """Pick and apply the fastest launch configuration for ``batch``; returns it."""
    key = _key(batch)
    path = cache_path()
    cache = {}
    if use_cache and path.exists():
        try:
            cache = json.loads(path.read_text())
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        cfg = cache[key]
        _apply(batch, cfg)
        return cfg
    if batch.store == nat.STORE_F64_EXACT:
        return {"kernel": "exact"}
    snap = _snapshot(batch)
    graph_steps = batch.graph_steps
    batch.graph_steps = 0
    results = []
    elem = batch.windows[0].f[0].element_size()
    tma_ok = all((w.nz * elem) % 16 == 0 and w.nz % 16 == 0 for w in batch.windows)
    sm = torch.cuda.get_device_properties(batch.device).multi_processor_count
    grids = (0, sm, 2 * sm, 4 * sm)  # 0: SM count x occupancy
    grid0 = batch.grid_ctas
    try:
        for cpt in (1, 2):
            for grid in (grids if cpt == 1 else (0,)):
                batch.configure(nat.KERNEL_DIRECT, cells_per_thread=cpt, grid_ctas=grid)
                results.append(({"kernel": "direct", "cells_per_thread": cpt, "grid_ctas": grid}, _time(batch, steps)))
                _restore(batch, snap)
        if all(w.nz % 2 == 0 for w in batch.windows):
            for grid in grids:
                batch.configure(nat.KERNEL_PAIR, grid_ctas=grid)
                results.append(({"kernel": "pair", "grid_ctas": grid}, _time(batch, steps)))
                _restore(batch, snap)
        batch.grid_ctas = grid0
        if tma_ok:
            # per size class: best rows (2 stages), timed on a batch of that class only
            classes = sorted({(w.nx, w.ny, w.nz) for w in batch.windows})
            best_rows = {}
            for cls in classes:
                idx = [k for k, w in enumerate(batch.windows) if (w.nx, w.ny, w.nz) == cls]
                sub = _SubBatch(batch, idx)
                timings = []
                for r in _row_candidates(cls[2], cls[1], elem, stages=2):
                    sub.configure(nat.KERNEL_TMA, rows_per_window=[r] * len(idx), stages=2)
                    timings.append((r, _time(sub, steps)))
                    _restore(batch, snap)
                best_rows[cls] = min(timings, key=lambda x: x[1])[0]
                if verbose:
                    print("class", cls, "rows timings", timings)
            rows = [best_rows[(w.nx, w.ny, w.nz)] for w in batch.windows]
            for stages in (2, 3, 4):
                if max(r * w.nz * (19 * elem + 1) for r, w in zip(rows, batch.windows)) * stages > 200 * 1024:
                    continue
                batch.configure(nat.KERNEL_TMA, rows_per_window=rows, stages=stages, grid_ctas=0)
                results.append(({"kernel": "tma", "stages": stages, "rows_per_window": rows, "grid_ctas": 0},
                                _time(batch, steps)))
                _restore(batch, snap)
    finally:
        batch.graph_steps = graph_steps
        batch.grid_ctas = grid0
    best = min(results, key=lambda x: x[1])
    cfg = dict(best[0])
    cfg["ms_per_step"] = best[1]
    cfg["candidates"] = [[c, t] for c, t in results]
    _apply(batch, cfg)
    _restore(batch, snap)
    if use_cache:
        cache[key] = cfg
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            path.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    if verbose:
        print("autotune:", cfg)
    return cfg


def _apply(batch, cfg: dict) -> None:
    grid = int(cfg.get("grid_ctas", 0))
    if cfg.get("kernel") == "tma":
        batch.configure(nat.KERNEL_TMA, stages=int(cfg["stages"]), rows_per_window=cfg["rows_per_window"],
                        grid_ctas=grid)
    elif cfg.get("kernel") == "direct":
        batch.configure(nat.KERNEL_DIRECT, cells_per_thread=int(cfg["cells_per_thread"]), grid_ctas=grid)
    elif cfg.get("kernel") == "pair":
        batch.configure(nat.KERNEL_PAIR, grid_ctas=grid)


class _SubBatch:
    """A view of some windows of a batch that can be stepped on its own (for class timing)."""

    def __init__(self, parent, idx):
        from .batch import PscBatch

        self._p = parent
        self.device = parent.device
        self._b = PscBatch.__new__(PscBatch)
        b = self._b
        b.device = parent.device
        b.store = parent.store
        b.precision = parent.precision
        b.graph_steps = 0
        b.grid_ctas = parent.grid_ctas
        b.specs = [parent.specs[k] for k in idx]
        b.windows = [parent.windows[k] for k in idx]
        b.geoms = [parent.geoms[k] for k in idx]
        b.cells = parent.cells[idx]
        b.parity = parent.parity
        b.steps_done = 1
        b.frozen = {}
        b._frozen_red = {}
        b._tables = None
        b._graphs = {}
        b._red = parent._red
        b.kernel = nat.KERNEL_TMA
        b.cells_per_thread = 1
        b.tile_rows = 0
        b.stages = 3
        b.stage_bytes = 0
        b.rows_per_window = None

    def configure(self, *a, **k):
        self._b.parity = self._p.parity
        self._b.configure(*a, **k)

    def run(self, steps):
        self._b.run(steps)
