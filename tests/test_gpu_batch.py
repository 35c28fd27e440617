"""Batched uneven windows: each window of a batch must evolve exactly as when solved alone.

The per-cell arithmetic does not depend on how cells are tiled or which
windows share a launch, so batched and solo populations agree bit for bit in
every storage mode; CUDA-graph replays must match direct launches.  FP64
reduction sums are grouped by each launch's CTA runs, so they agree to
rounding.
"""

import numpy as np
import pytest

from oracle import psc_oracle as orc

pytestmark = pytest.mark.gpu


def small_windows():
    from particuology_hydraulic_penalty_b200 import windows as wgen

    return [wgen.make_window(24, "skeleton", 1), wgen.make_window(32, "passive", 2),
            wgen.make_window(40, "preloaded", 3)]


@pytest.mark.parametrize("precision", ["fp64-exact", "fp32", "fp16"])
def test_batched_equals_solo(precision):
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = small_windows()
    specs = [WindowSpec(w.n, w.particles, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4) for w in wins]
    batch = PscBatch(specs, precision=precision, graph_steps=4)
    batch.run(11)  # warm step + 2 graph replays + 2 direct steps
    kb = batch.permeability()
    fields_b = [batch.velocity_field(k) for k in range(len(wins))]
    for k, spec in enumerate(specs):
        solo = PscBatch([spec], precision=precision, graph_steps=0)
        solo.run(11)
        # FP64 reduction rows are grouped by the launch's CTA runs: equal to rounding
        assert abs(solo.permeability()[0] - kb[k]) <= 1e-12 * abs(kb[k])
        assert np.array_equal(solo.velocity_field(0), fields_b[k])


def test_batch_exact_matches_oracle():
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    w = small_windows()[1]
    spec = WindowSpec(w.n, w.particles, tau=0.8, force=(0.0, 0.0, 2e-6), subsamples=2)
    batch = PscBatch([spec], precision="fp64-exact", graph_steps=2)
    batch.run(4)
    o = orc.OracleSolver(w.n, w.particles, tau=0.8, subsamples=2, body_force_z=2e-6, static_geometry=True)
    for _ in range(4):
        o.collide_stream_psc()
    mom = batch.velocity_field(0)
    assert np.array_equal(mom[3], o.uz)
    assert np.array_equal(mom[0], o.rho)
    k = orc.darcy_permeability(o.solid, o.uz, 0.8, 2e-6)["permeability_lu"]
    assert abs(batch.permeability()[0] - k) <= 1e-13 * abs(k)


def test_batch_loads_match_dropin():
    from particuology_hydraulic_penalty_b200 import SparsePscD3Q19
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    w = small_windows()[2]
    spec = WindowSpec(w.n, w.particles, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4)
    batch = PscBatch([spec], precision="fp32", graph_steps=0)
    batch.run(5)
    F, T = batch.loads()[0]
    s = SparsePscD3Q19(w.n, w.particles, tau=0.8, subsamples=4, static_geometry=True, precision="fp32",
                       force=(1e-6, 0.0, 0.0))
    for _ in range(6):
        s.collide_stream_psc()
    # the drop-in reduces from its loads list, this batch over the whole boxes: the same sums in
    # another order, equal to round-off
    assert np.linalg.norm(F - s.hydro_forces) <= 1e-12 * np.linalg.norm(s.hydro_forces)
    assert np.linalg.norm(T - s.hydro_torques) <= 1e-12 * np.linalg.norm(s.hydro_torques)


@pytest.mark.parametrize("precision", ["fp32", "fp64", "bf16"])
def test_cells_per_thread_variants_identical(precision):
    """The multi-cell thread variants run the same per-cell arithmetic: bit-identical fields."""
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = small_windows()
    specs = [WindowSpec(w.n, w.particles, tau=0.8, force=(1e-6, 2e-7, 0.0), subsamples=4) for w in wins]
    ref = None
    for cpt in (1, 2, 4):
        b = PscBatch(specs, precision=precision, graph_steps=0, cells_per_thread=cpt)
        b.run(7)
        fields = [b.velocity_field(k) for k in range(len(wins))]
        red = b.observe()
        if ref is None:
            ref = (fields, red)
        else:
            for a, c in zip(fields, ref[0]):
                assert np.array_equal(a, c)
            # per-tile FP64 partials group cells differently: equal to round-off
            assert np.allclose(red, ref[1], rtol=1e-13, atol=1e-13 * np.abs(ref[1]).max())


@pytest.mark.parametrize("precision", ["fp32", "fp64", "fp16"])
@pytest.mark.parametrize("rows", [0, 3])
def test_tma_kernel_matches_direct(precision, rows):
    """The TMA-staged kernel computes the same per-cell arithmetic as the direct one."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    from particuology_hydraulic_penalty_b200 import windows as wgen

    # row tiles carry the uint8 level by bulk copy: nz must be a multiple of 16
    wins = [wgen.make_window(16, "skeleton", 1), wgen.make_window(32, "passive", 2),
            wgen.make_window(48, "preloaded", 3)]
    specs = [WindowSpec(w.n, w.particles, tau=0.8, force=(1e-6, 0.0, 3e-7), subsamples=4) for w in wins]
    d = PscBatch(specs, precision=precision, graph_steps=0)
    d.run(9)
    t = PscBatch(specs, precision=precision, graph_steps=4, kernel=nat.KERNEL_TMA, tile_rows=rows, stages=3)
    t.run(9)
    for k in range(len(wins)):
        assert np.array_equal(t.velocity_field(k), d.velocity_field(k))
    rd, rt = d.observe(), t.observe()
    assert np.allclose(rt, rd, rtol=1e-13, atol=1e-13 * np.abs(rd).max())
    status = ctypes_status()
    assert status == 0


def ctypes_status():
    import ctypes

    from particuology_hydraulic_penalty_b200 import _native as nat

    v = ctypes.c_int(0)
    nat.call("psc_device_status", ctypes.byref(v), 1)
    return v.value


def test_tma_kernel_with_reductions_and_loads():
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    w = small_windows()[1]
    spec = WindowSpec(w.n, w.particles, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4)
    d = PscBatch([spec], precision="fp32", graph_steps=0)
    t = PscBatch([spec], precision="fp32", graph_steps=0, kernel=nat.KERNEL_TMA, stages=2)
    d.run(4)
    t.run(4)
    Fd, Td = d.loads()[0]
    Ft, Tt = t.loads()[0]
    assert np.array_equal(Fd, Ft) and np.array_equal(Td, Tt)
    assert ctypes_status() == 0


@pytest.mark.parametrize("kernel", ["direct", "tma"])
def test_converged_windows_freeze_exactly(kernel):
    """A window frozen at convergence keeps exactly the state it had at its convergence step."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    k = {"direct": nat.KERNEL_DIRECT, "tma": nat.KERNEL_TMA}[kernel]
    wins = [wgen.make_window(16, "skeleton", 4), wgen.make_window(32, "passive", 5), wgen.make_window(48, "preloaded", 6)]
    specs = [WindowSpec(w.n, w.particles, tau=0.9, force=(1e-5, 0.0, 0.0), subsamples=2) for w in wins]
    b = PscBatch(specs, precision="fp32", graph_steps=4, kernel=k)
    res = b.run_to_convergence(tol=1e-5, check_every=40, max_steps=4000)
    assert res["converged"].all()
    assert len(set(res["steps"].tolist())) > 1  # windows converge at different steps
    kb = b.permeability()
    for j, spec in enumerate(specs):
        solo = PscBatch([spec], precision="fp32", graph_steps=0, kernel=k)
        solo.run(int(res["steps"][j]))
        assert abs(solo.permeability()[0] - kb[j]) <= 1e-12 * abs(kb[j])
        assert np.array_equal(solo.velocity_field(0), b.velocity_field(j))
    assert ctypes_status() == 0


@pytest.mark.parametrize("kernel", ["direct", "tma"])
def test_trt_matches_oracle(kernel):
    """TRT (magic 3/16) on the GPU in FP64 against the oracle's TRT extension, 6 steps."""
    from oracle import psc_oracle as orc
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec
    from particuology_hydraulic_penalty_b200.engine import trt_tau_minus

    w = small_windows()[1]
    tau, F = 0.8, (1e-5, 0.0, 3e-6)
    spec = WindowSpec(w.n, w.particles, tau=tau, force=F, subsamples=2, collision="trt")
    k = {"direct": nat.KERNEL_DIRECT, "tma": nat.KERNEL_TMA}[kernel]
    b = PscBatch([spec], precision="fp64", graph_steps=0, kernel=k)
    b.run(6)
    geo = orc.voxelize(w.particles, w.n, 2)
    g = np.zeros((19,) + (w.n,) * 3)
    S = g
    for _ in range(6):
        S = orc.collide_trt_deviation(orc.stream_push(S), geo.solid, tau, trt_tau_minus(tau), F)
    f = orc.stream_push(S)
    rho = 1.0 + f.sum(axis=0)
    ux = (np.einsum("i,i...->...", orc.C[:, 0].astype(float), f) + 0.5 * F[0]) / rho
    mom = b.velocity_field(0)
    assert np.abs(mom[1] - ux).max() <= 1e-12 * np.abs(ux).max()
    # TRT differs from BGK on the same window
    bb = PscBatch([WindowSpec(w.n, w.particles, tau=tau, force=F, subsamples=2)], precision="fp64", graph_steps=0)
    bb.run(6)
    assert np.abs(bb.velocity_field(0)[1] - mom[1]).max() > 1e-3 * np.abs(ux).max()


@pytest.mark.parametrize("precision", ["fp32", "fp64", "fp16", "bf16"])
def test_pair_kernel_matches_direct(precision):
    """Two cells per thread with paired loads/stores: the same arithmetic per cell, identical populations."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = [wgen.make_window(16, "skeleton", 1), wgen.make_window(26, "passive", 2),
            wgen.make_window(48, "preloaded", 3)]
    moving = wins[1].particles.copy()
    moving[:, 4:7] = 2e-4  # the moving-particle path too
    specs = [WindowSpec(wins[0].n, wins[0].particles, tau=0.8, force=(1e-6, 0.0, 3e-7), subsamples=4),
             WindowSpec(wins[1].n, moving, tau=0.7, force=(0.0, 2e-6, 0.0), subsamples=4, collision="trt"),
             WindowSpec(wins[2].n, wins[2].particles, tau=0.9, force=(0.0, 0.0, 0.0), subsamples=4,
                        inlet=(1.0, (0.003, 0.0, 0.0005)))]
    d = PscBatch(specs, precision=precision, graph_steps=0)
    d.run(9)
    p = PscBatch(specs, precision=precision, graph_steps=4, kernel=nat.KERNEL_PAIR)
    p.run(9)
    for k in range(len(specs)):
        assert np.array_equal(p.velocity_field(k), d.velocity_field(k))
        assert np.array_equal(p.windows[k].post_stream_f().cpu().numpy(), d.windows[k].post_stream_f().cpu().numpy())
    rd, rp = d.observe(), p.observe()
    assert np.allclose(rp, rd, rtol=1e-13, atol=1e-13 * np.abs(rd).max())
    Fd, Td = d.loads()[1]
    Fp, Tp = p.loads()[1]
    assert np.array_equal(Fd, Fp) and np.array_equal(Td, Tp)
    assert ctypes_status() == 0
