"""The accuracy gate of FP32 deviation storage: Darcy permeability within 1e-4 relative of the FP64
form (FP64 deviation storage, itself within 1e-10 of the reference's arithmetic on the golden runs).

* the packed-bed case (one seeded 96^3 window in its skeleton / passive-fines / preloaded geometries,
  S = 4, tau = 0.8, F = 1e-6 along x), each precision run to its own steady state with the reference
  coupled driver's criterion (relative change between consecutive steps < 1e-8,
  coupling_sync/couple_psc_liggghts.py:284-296), K as in run_psc_permeability_resolution.py:144-150;
* the 24-window benchmark batch at equal step counts from rest;
* the high-resolution preloaded windows (192^3 and 256^3) at equal step counts.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOUND = 1e-4


def _specs(wins, force=(1.0e-6, 0.0, 0.0)):
    from particuology_hydraulic_penalty_b200.batch import WindowSpec

    return [WindowSpec(w.n, w.particles, 0.8, force, 4, name=getattr(w, "kind", "")) for w in wins]


def _equal_steps(specs, steps):
    from particuology_hydraulic_penalty_b200.batch import PscBatch

    K = {}
    for prec in ("fp64", "fp32"):
        b = PscBatch(specs, precision=prec, graph_steps=20)
        b.run(steps)
        assert b.steps_done == steps
        red = b.observe()
        assert not b.nonfinite(red).any()
        K[prec] = b.permeability(red)
        del b
    return K


def test_packed_bed_fp32_steady_state_within_bound():
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.batch import PscBatch

    wins = [wgen.make_window(96, kind, 1000) for kind in wgen.GEOMETRY_TYPES]
    res = {}
    for prec in ("fp64", "fp32"):
        b = PscBatch(_specs(wins), precision=prec, graph_steps=20)
        res[prec] = b.run_to_convergence(tol=1.0e-8, check_every=200, max_steps=100000)
        del b
    for prec in res:
        assert res[prec]["converged"].all(), (prec, res[prec]["residual"])
    k64, k32 = res["fp64"]["permeability"], res["fp32"]["permeability"]
    assert np.all(k64 > 0.0)
    err = np.abs(k32 - k64) / np.abs(k64)
    assert err.max() <= BOUND, err


def test_benchmark_batch_fp32_equal_steps_within_bound():
    import bench

    wins = bench.make_windows("batch24", 0)
    K = _equal_steps(_specs(wins, bench.FORCE), 1000)
    err = np.abs(K["fp32"] - K["fp64"]) / np.abs(K["fp64"])
    assert err.max() <= BOUND, err


@pytest.mark.parametrize("n", [192, 256])
def test_high_resolution_preloaded_fp32_equal_steps_within_bound(n):
    from particuology_hydraulic_penalty_b200 import windows as wgen

    w = wgen.make_window(n, "preloaded", 1000)
    K = _equal_steps(_specs([w]), 2000)
    err = abs(K["fp32"][0] - K["fp64"][0]) / abs(K["fp64"][0])
    assert K["fp64"][0] > 0.0
    assert err <= BOUND, err
