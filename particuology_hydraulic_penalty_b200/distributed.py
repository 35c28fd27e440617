"""Window-parallel runs over several GPUs (one process per GPU).

Pore windows are independent: nothing crosses a window boundary during a
step, so N GPUs solve disjoint window sets with no per-step collective.  The
only exchange is one gather of the per-window results (permeability, flux,
porosity, particle loads) after the run.  Windows are assigned by longest
processing time first, cost = cells x steps, so uneven window sizes balance.

The reference has no parallelism beyond a process pool for voxelisation and
one process per campaign row (coupling_sync/run_synced_campaign.py:242);
this is the GPU counterpart of that campaign-level split.
"""

from __future__ import annotations

import heapq
from typing import Callable, Sequence

import numpy as np


def partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of items to ``world`` ranks.

    Deterministic (ties by index), every rank gets a sorted index list.
    """
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(x) for x in out]


def window_costs(cells: Sequence[int], steps: Sequence[int] | int) -> np.ndarray:
    cells = np.asarray(cells, dtype=np.float64)
    steps = np.broadcast_to(np.asarray(steps, dtype=np.float64), cells.shape)
    return cells * steps


def run_partitioned(items: Sequence, costs: Sequence[float], solve: Callable[[list], list],
                    group=None) -> list | None:
    """Solve ``items`` across the ranks of ``group``; rank 0 returns all results in item order.

    ``solve(list_of_items) -> list_of_results`` runs on each rank for its own
    share (on that rank's GPU).  Results must be picklable; other ranks
    return None.  Every rank takes the same collective steps (one
    gather_object), also when its share is empty.
    """
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return list(solve(list(items)))
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = partition(costs, world)
    mine = parts[rank]
    local = list(solve([items[i] for i in mine])) if mine else []
    if len(local) != len(mine):
        raise RuntimeError(f"rank {rank}: solve returned {len(local)} results for {len(mine)} items")
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, local)), gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(items)
    for chunk in gathered:
        for i, res in chunk:
            out[i] = res
    return out


def batch_solver(precision: str = "fp32", steps: int = 1000, graph_steps: int = 20) -> Callable[[list], list]:
    """A ``solve`` for :func:`run_partitioned`: one PscBatch per rank, per-window Darcy K."""

    def solve(specs: list) -> list:
        from .batch import PscBatch

        b = PscBatch(specs, precision=precision, graph_steps=graph_steps)
        b.run(steps)
        red = b.observe()
        k = b.permeability(red)
        return [{"permeability_lu": float(k[i]), "porosity": float(red[i, 7] / b.cells[i]),
                 "nonfinite": bool(red[i, 11] > 0)} for i in range(len(specs))]

    return solve
