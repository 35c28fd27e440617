"""Window-parallel host logic with world_size 2 on CPU (gloo)."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from particuology_hydraulic_penalty_b200 import distributed as pd


def test_partition_balances_and_covers():
    costs = [48 ** 3, 64 ** 3, 96 ** 3, 128 ** 3, 160 ** 3, 48 ** 3, 160 ** 3, 96 ** 3]
    parts = pd.partition(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    # LPT is within 4/3 of the optimum; the optimum is at least the mean load
    assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / 3, max(costs)) + 1
    assert pd.partition(costs, 3) == parts  # deterministic


def test_partition_more_ranks_than_items():
    parts = pd.partition([5.0, 3.0], 4)
    assert sorted(len(p) for p in parts) == [0, 0, 1, 1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, results):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    items = list(range(7))
    costs = [1, 9, 3, 3, 8, 2, 5]

    def solve(chunk):
        # stands in for the GPU batch solve: a deterministic function of the item
        return [{"item": i, "rank": rank, "k": 0.5 * i} for i in chunk]

    out = pd.run_partitioned(items, costs, solve)
    if rank == 0:
        results.put(out)
    else:
        results.put(None if out is None else "bad")
    dist.barrier()
    dist.destroy_process_group()


def test_run_partitioned_gathers_in_order():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = [g for g in got if isinstance(g, list)]
    assert len(full) == 1 and got.count(None) == 1
    out = full[0]
    assert [r["item"] for r in out] == list(range(7))
    assert all(r["k"] == 0.5 * r["item"] for r in out)
    ranks = {r["rank"] for r in out}
    assert ranks == {0, 1}


def test_run_partitioned_without_process_group():
    out = pd.run_partitioned([1, 2, 3], [1, 1, 1], lambda xs: [x * 2 for x in xs])
    assert out == [2, 4, 6]


def test_window_costs():
    c = pd.window_costs([8, 27], 10)
    assert np.array_equal(c, [80.0, 270.0])
