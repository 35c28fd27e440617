"""bench.py's multi-rank path on CPU: ``--gpus N`` without torchrun starts N local ranks with the
torchrun environment, the ranks reduce their timings (max) and cells (sum) over a process group, and
rank 0 alone prints the JSON line.  The GPU solve is replaced by a stub; the process group is gloo."""

import json
import subprocess
import sys
import textwrap
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

# one rank: the bench's own set-up and reductions around a stand-in for the batch solve
RANK_STUB = textwrap.dedent("""
    import json, os, sys
    sys.path.insert(0, {root!r})
    import bench
    world, rank, local = bench.dist_setup(backend="gloo")
    assert int(os.environ["LOCAL_RANK"]) == local == rank
    assert os.environ["MASTER_ADDR"] == "127.0.0.1"
    ms = 10.0 + rank            # the rank's timed region
    cells = 1000 * (rank + 1)   # the rank's cells
    ms_max = bench.max_over_ranks(ms, world)
    cells_all = bench.sum_over_ranks(float(cells), world)
    if rank == 0:
        print(json.dumps({{"n_gpus": world, "ms_max": ms_max, "cells_all": cells_all}}), flush=True)
    else:
        print("rank output must not reach stdout", flush=True)
    import torch.distributed as dist
    dist.barrier()
    dist.destroy_process_group()
    sys.exit({exit_code})
""")


def _launch(n, exit_code_of_rank1=0):
    stub = RANK_STUB.format(root=str(ROOT), exit_code="0 if rank != 1 else %d" % exit_code_of_rank1)
    driver = textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {str(ROOT)!r})
        import bench
        sys.exit(bench.spawn_ranks({n}, [sys.executable, "-c", {stub!r}], timeout_s=120))
    """)
    return subprocess.run([sys.executable, "-c", driver], capture_output=True, text=True, timeout=180)


def test_two_ranks_reduce_and_rank0_prints_once():
    p = _launch(2)
    assert p.returncode == 0, p.stderr
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, p.stdout
    out = json.loads(lines[0])
    assert out == {"n_gpus": 2, "ms_max": 11.0, "cells_all": 3000.0}


def test_failing_rank_sets_exit_code():
    p = _launch(2, exit_code_of_rank1=3)
    assert p.returncode == 3, (p.returncode, p.stderr)


def test_bench_gpus2_reference_arm_spawns_ranks():
    """``bench.py --impl reference --gpus 2`` outside torchrun: two ranks start, rank 1 exits without
    work, rank 0 prints the one reference line (a one-step sample of the CPU reference path)."""
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert p.returncode == 0, p.stderr
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, p.stdout
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["value"] > 0.0
    assert out["e2e"]["h2d_bytes_per_step"] == 0


# one rank of the end-to-end leg: the batch handle replaced by a stand-in (no GPU)
E2E_STUB = textwrap.dedent("""
    import json, sys, types
    import numpy as np
    sys.path.insert(0, {root!r})
    import bench
    from particuology_hydraulic_penalty_b200 import handle

    class FakeBatch:
        calls = 0
        def __init__(self, cfgs, graph_steps=0):
            self.n = len(cfgs)
        def set_particles(self, k, arr):
            pass
        def set_particles_all(self, arrays):
            assert len(arrays) == self.n
        def step(self, nsteps, flags=0):
            FakeBatch.calls += 1
            d = types.SimpleNamespace(permeability=1.0)
            return [types.SimpleNamespace(diag=d)]
        def close(self):
            pass

    handle.BatchHandle = FakeBatch
    world, rank, local = bench.dist_setup(backend="gloo")
    wins = [types.SimpleNamespace(n=8 + 8 * rank, particles=np.zeros((3 + rank, 10)))]
    out = bench.run_e2e_batch(wins, steps=4, graph_steps=0, world=world)
    if rank == 0:
        print(json.dumps(out), flush=True)
    import torch.distributed as dist
    dist.barrier()
    dist.destroy_process_group()
""")


def test_e2e_leg_runs_on_every_rank():
    """Each rank runs its own batch through the (stand-in) C ABI; cells and copied bytes add up over
    the ranks and the rate uses the slowest rank's wall time."""
    stub = E2E_STUB.format(root=str(ROOT))
    driver = textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {str(ROOT)!r})
        import bench
        sys.exit(bench.spawn_ranks(2, [sys.executable, "-c", {stub!r}], timeout_s=120))
    """)
    p = subprocess.run([sys.executable, "-c", driver], capture_output=True, text=True, timeout=180)
    assert p.returncode == 0, p.stderr
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, p.stdout
    out = json.loads(lines[0])
    assert out["ranks"] == 2 and out["finite"] is True
    assert out["h2d_bytes_per_step"] == (3 + 4) * 10 * 8
    assert out["value"] > 0.0
