"""Properties that hold at any size, checked at the benchmark's full sizes and
at the largest window the 32-bit population offsets allow (fewer than
2^31 / 19 cells): uniform acceleration of an empty window, batched == solo
on the 24-window batch, Darcy linearity, mass conservation and momentum
closure on the 96^3 windows."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_largest_window_accelerates_uniformly():
    """n = 482 (111.98 M cells, 19 N < 2^31): no particles, body force F along x.  Every cell runs the
    same arithmetic, so the field stays bitwise uniform.  With the reference's forcing (u_eff carries F/2
    twice, psc3d.py:214-219, and the Guo term adds (1 - 1/2tau) F) the momentum grows by
    F (1 + 1/(2 tau)) per step, and the reported u_x = (m + F/2) / rho: an offset that overflowed would
    break both."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.handle import SolverHandle, make_config

    n, F, steps = 482, 1e-6, 4
    assert 19 * n ** 3 < 2 ** 31
    h = SolverHandle(make_config((n, n, n), tau=0.8, force=(F, 0.0, 0.0), subsamples=2, store=nat.STORE_F32))
    h.set_particles(np.zeros((0, 10)))
    st = h.step(steps, nat.RUN_DIAG)
    ux = h.field(nat.FIELD_UX)
    assert np.ptp(ux) == 0.0
    expect = (steps * (1.0 + 0.5 / 0.8) + 0.5) * F  # the oracle gives the same for any lattice size
    assert abs(ux[0] - expect) <= 1e-4 * expect
    assert st.diag.nonfinite_cells == 0
    assert abs(st.diag.mean_u[0] - ux[0]) <= 1e-6 * abs(ux[0])
    h.close()


def test_full_batch_equals_solo():
    """The 24-window benchmark batch (edges 48-160, 33 M cells) at full size: batched windows evolve
    exactly as when solved alone (the largest and a small one)."""
    import bench
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = bench.make_windows("batch24", 0)
    specs = [WindowSpec(w.n, w.particles, bench.TAU, bench.FORCE, bench.SUBSAMPLES) for w in wins]
    b = PscBatch(specs, precision="fp32", graph_steps=10)
    b.run(20)
    big = int(np.argmax([w.n for w in wins]))
    small = int(np.argmin([w.n for w in wins]))
    fields = {k: b.velocity_field(k) for k in (big, small)}
    del b
    for k in (big, small):
        solo = PscBatch([specs[k]], precision="fp32", graph_steps=0)
        solo.run(20)
        assert np.array_equal(solo.velocity_field(0), fields[k])


def test_config2_linearity_mass_and_closure():
    """The three 96^3 geometries (FP32): Darcy K is linear in the body force at these Reynolds
    numbers, mass is conserved, and the particle forces balance the node IMB momentum."""
    from particuology_hydraulic_penalty_b200 import SparsePscD3Q19
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = [wgen.make_window(96, kind, 1000) for kind in wgen.GEOMETRY_TYPES]
    K = []
    for F in (1e-6, 2e-6):
        b = PscBatch([WindowSpec(w.n, w.particles, 0.8, (F, 0.0, 0.0), 4) for w in wins], precision="fp32",
                     graph_steps=20)
        b.run(400)
        red = b.observe()
        K.append(b.permeability(red))
        rho_mean = red[:, 0] / np.array([w.n ** 3 for w in wins])
        assert np.all(np.abs(rho_mean - 1.0) <= 1e-5)
    assert np.all(np.abs(K[1] / K[0] - 1.0) <= 1e-2)
    w = wins[2]  # preloaded fines
    s = SparsePscD3Q19(w.n, w.particles, tau=0.8, subsamples=4, static_geometry=True, precision="fp32",
                       force=(1e-6, 0.0, 0.0))
    for _ in range(30):
        d = s.collide_stream_psc()
    total = float(np.abs(s.hydro_forces).sum())
    assert total > 0.0
    assert d["momentum_residual"] <= 1e-9 * total


def test_batch24_5000_steps_permeability_equals_solo():
    """The batched-windows configuration at its stated length: the 24 seeded windows (edges 48-160,
    FP32, one persistent launch per step from CUDA graphs) run 5000 steps, and every window's Darcy
    permeability equals that of the window run alone for 5000 steps (the populations evolve bit for
    bit alike; the FP64 window sums group their partial rows differently, hence 1e-12)."""
    import bench
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    steps = 5000
    wins = bench.make_windows("batch24", 0)
    specs = [WindowSpec(w.n, w.particles, bench.TAU, bench.FORCE, bench.SUBSAMPLES) for w in wins]
    b = PscBatch(specs, precision="fp32", graph_steps=20)
    b.run(steps)
    K = b.permeability(b.observe())
    del b
    assert np.all(np.isfinite(K)) and np.all(K > 0.0)
    for k, spec in enumerate(specs):
        solo = PscBatch([spec], precision="fp32", graph_steps=20)
        solo.run(steps)
        Ks = solo.permeability(solo.observe())[0]
        del solo
        assert abs(Ks - K[k]) <= 1e-12 * abs(Ks), (k, Ks, K[k])
