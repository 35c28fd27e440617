"""The handle layer (psc_solver / psc_batch): multi-step calls, the
lbm_converge criterion run natively, and batches of windows behind one
handle must reproduce the oracle and the single-step / Python-side paths
exactly."""

import numpy as np
import pytest

from oracle import psc_oracle as orc
from tests import golden_io

pytestmark = pytest.mark.gpu


def _window(n=24, kind="passive", seed=5):
    from particuology_hydraulic_penalty_b200 import windows as wgen

    return wgen.make_window(n, kind, seed)


def _solver(w, precision="fp64-exact", static=True, force=(0.0, 0.0, 2e-6), subsamples=2, tau=0.8, **kw):
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.engine import store_mode
    from particuology_hydraulic_penalty_b200.handle import SolverHandle, make_config

    cfg = make_config((w.n,) * 3, tau=tau, force=force, subsamples=subsamples, store=store_mode(precision),
                      static_geometry=static, **kw)
    h = SolverHandle(cfg)
    h.set_particles(w.particles)
    return h, nat


def test_fields_before_first_step():
    w = _window(16)
    h, nat = _solver(w)
    assert np.all(h.field(nat.FIELD_RHO) == 1.0)
    assert np.all(h.field(nat.FIELD_UZ) == 0.0)
    assert np.all(h.field(nat.FIELD_SOLID) == 0.0)  # nothing voxelised yet (psc3d.py:144)
    F, T = h.loads()
    assert not F.any() and not T.any()


def test_multi_step_call_matches_oracle_bitwise():
    w = _window()
    h, nat = _solver(w)
    st = h.step(6, nat.RUN_DIAG)
    assert st.steps_done == 6
    o = orc.OracleSolver(w.n, w.particles, tau=0.8, subsamples=2, body_force_z=2e-6, static_geometry=True)
    for _ in range(6):
        d = o.collide_stream_psc()
    shape = (w.n,) * 3
    assert np.array_equal(h.field(nat.FIELD_F).reshape((19, *shape)), o.f)
    assert np.array_equal(h.field(nat.FIELD_UZ).reshape(shape), o.uz)
    assert np.array_equal(h.field(nat.FIELD_SOLID).reshape(shape), o.solid)
    assert abs(st.diag.mean_uz - d["mean_uz"]) <= 1e-14 * abs(d["mean_uz"])
    F, T = h.loads()
    assert np.linalg.norm(F - o.hydro_forces) <= 1e-12 * np.linalg.norm(o.hydro_forces)
    # Darcy K of the diagnostics (run_psc_permeability_resolution.py:144-150)
    k = orc.darcy_permeability(o.solid, o.uz, 0.8, 2e-6)["permeability_lu"]
    assert abs(st.diag.permeability - k) <= 1e-12 * abs(k)


def test_converge_flag_matches_python_loop():
    """PSC_RUN_CONVERGE stops where lbm_converge (couple_psc_liggghts.py:284-296) stops."""
    from particuology_hydraulic_penalty_b200 import SparsePscD3Q19
    from particuology_hydraulic_penalty_b200.coupling import lbm_converge

    w = _window(20, "skeleton", 7)
    tol = 1e-2
    h, nat = _solver(w, precision="fp32", subsamples=3, conv_tol=tol, conv_min_steps=3)
    st = h.step(400, nat.RUN_CONVERGE)
    s = SparsePscD3Q19(w.n, w.particles, tau=0.8, subsamples=3, body_force_z=2e-6, static_geometry=True,
                       precision="fp32")
    it, res, ok, diag = lbm_converge(s, residual_tol=tol, min_steps=3, max_steps=400)
    assert ok and st.converged == 1
    assert st.steps_done == it
    assert st.residual == res
    assert st.diag.mean_uz == diag["mean_uz"]
    assert st.diag.momentum_residual == diag["momentum_residual"]
    assert np.array_equal(h.field(nat.FIELD_F), s.f.reshape(-1))


def test_moving_nonstatic_rebuilds_like_oracle():
    """Particles moved between calls of a non-static solver: voxelised again, bit for bit."""
    w = _window(20, "preloaded", 9)
    parts = w.particles.copy()
    parts[:, 4] = 1e-3
    h, nat = _solver(w, static=False)
    o = orc.OracleSolver(w.n, parts, tau=0.8, subsamples=2, body_force_z=2e-6, static_geometry=False)
    for step in range(3):
        moved = parts.copy()
        moved[:, 0] += 0.37 * step
        h.set_particles(moved)
        o.particles = moved
        h.step(1, nat.RUN_DIAG)
        o.collide_stream_psc()
    shape = (w.n,) * 3
    assert np.array_equal(h.field(nat.FIELD_SOLID).reshape(shape), o.solid)
    assert np.array_equal(h.field(nat.FIELD_F).reshape((19, *shape)), o.f)
    us = np.stack([h.field(nat.FIELD_US_X + k).reshape(shape) for k in range(3)])
    assert np.array_equal(us, orc.solid_velocity(o.particles, o.geo))


def test_accumulate_and_populations_roundtrip():
    w = _window(16, "skeleton", 3)
    h, nat = _solver(w, subsamples=3)
    h.step(2, 0)
    F0, T0 = h.loads()
    h.accumulate_loads()
    F1, T1 = h.loads()
    assert np.array_equal(F0, F1) and np.array_equal(T0, T1)
    f = h.field(nat.FIELD_F)
    h.set_populations(f)
    assert np.array_equal(h.field(nat.FIELD_F), f)


def _batch(wins, precision="fp32", launch=None, graph_steps=4):
    from particuology_hydraulic_penalty_b200.engine import store_mode
    from particuology_hydraulic_penalty_b200.handle import BatchHandle, make_config

    cfgs = [make_config((w.n,) * 3, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4, store=store_mode(precision))
            for w in wins]
    b = BatchHandle(cfgs, launch=launch, graph_steps=graph_steps)
    for k, w in enumerate(wins):
        b.set_particles(k, w.particles)
    return b


def _three():
    return [_window(24, "skeleton", 1), _window(32, "passive", 2), _window(40, "preloaded", 3)]


@pytest.mark.parametrize("precision", ["fp64-exact", "fp32", "fp16"])
def test_batch_handle_matches_python_batch(precision):
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = _three()
    b = _batch(wins, precision)
    st = b.step(11, nat.RUN_DIAG)  # graph replays + direct steps + the reporting step
    py = PscBatch([WindowSpec(w.n, w.particles, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4) for w in wins],
                  precision=precision, graph_steps=4)
    py.run(10)
    loads = py.loads()  # one more step with IMB
    red = py.observe()
    K = py.permeability(red)
    for k, w in enumerate(wins):
        assert st[k].steps_done == 11
        assert st[k].diag.permeability == K[k]
        mom = py.velocity_field(k)
        assert np.array_equal(b.field(k, nat.FIELD_UX), mom[1].reshape(-1).astype(np.float64))
        F, T = b.loads(k)
        # the handle reduces from its loads list, PscBatch over the whole boxes: equal to round-off
        assert np.linalg.norm(F - loads[k][0]) <= 1e-12 * np.linalg.norm(loads[k][0])
        assert np.linalg.norm(T - loads[k][1]) <= 1e-12 * np.linalg.norm(loads[k][1])


def test_batch_handle_tma_matches_direct():
    from particuology_hydraulic_penalty_b200 import _native as nat

    # bulk copies of the uint8 level rows need nz % 16 == 0
    wins = [_window(32, "skeleton", 1), _window(48, "passive", 2), _window(32, "preloaded", 3)]
    direct = _batch(wins)
    tma = _batch(wins, launch=nat.PscLaunch(0, 1, nat.KERNEL_TMA, 3, 0))
    direct.step(9, nat.RUN_DIAG)
    tma.step(9, nat.RUN_DIAG)
    for k in range(len(wins)):
        assert np.array_equal(direct.field(k, nat.FIELD_F), tma.field(k, nat.FIELD_F))
        # row tiles group the FP64 partial sums differently from 256-cell tiles
        kd, kt = direct.diag(k).permeability, tma.diag(k).permeability
        assert abs(kd - kt) <= 1e-12 * abs(kd)


def test_batch_handle_converge_matches_python():
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = _three()
    b = _batch(wins, graph_steps=10)
    st = b.converge(tol=1e-4, check_every=50, max_steps=3000)
    py = PscBatch([WindowSpec(w.n, w.particles, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4) for w in wins],
                  precision="fp32", graph_steps=10)
    res = py.run_to_convergence(tol=1e-4, check_every=50, max_steps=3000)
    assert res["converged"].any()
    for k in range(len(wins)):
        assert bool(st[k].converged) == bool(res["converged"][k])
        if res["converged"][k]:
            assert st[k].steps_done == int(res["steps"][k])
        assert st[k].diag.permeability == res["permeability"][k]


def test_batch_set_particles_all_equals_per_window():
    from particuology_hydraulic_penalty_b200 import _native as nat

    wins = _three()
    a = _batch(wins)
    b = _batch(wins)
    moved = [w.particles.copy() for w in wins]
    for m in moved:
        m[:, 0] += 0.25
    for k, m in enumerate(moved):
        a.set_particles(k, m)
    b.set_particles_all(moved)
    a.step(3, nat.RUN_DIAG)
    b.step(3, nat.RUN_DIAG)
    for k in range(len(wins)):
        assert np.array_equal(a.field(k, nat.FIELD_F), b.field(k, nat.FIELD_F))
        assert np.array_equal(a.loads(k)[0], b.loads(k)[0])


def test_batch_loads_one_launch_match_solo_windows():
    """The batch computes the loads of all its windows in one launch sequence (one chunk space over
    every window).  Windows with different sub-sample counts (the per-block count / S^3 table is
    rebuilt when S changes), one without particles, and uneven sizes: forces, torques and the
    load diagnostics equal those of each window solved alone."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.handle import BatchHandle, SolverHandle, make_config

    wins = [_window(24, "skeleton", 1), _window(32, "passive", 2), None, _window(40, "preloaded", 3),
            _window(24, "passive", 4)]
    sizes = [24, 32, 16, 40, 24]
    subs = [4, 3, 2, 4, 2]
    parts = [w.particles if w is not None else np.zeros((0, 10)) for w in wins]
    cfgs = [make_config((n,) * 3, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=s, store=nat.STORE_F32)
            for n, s in zip(sizes, subs)]
    b = BatchHandle(cfgs, graph_steps=4)
    b.set_particles_all(parts)
    b.step(7, nat.RUN_DIAG)
    for rep in range(2):  # a second reporting step reuses the uploaded job table
        for k in range(len(cfgs)):
            h = SolverHandle(make_config((sizes[k],) * 3, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=subs[k],
                                         store=nat.STORE_F32))
            h.set_particles(parts[k])
            h.step(7 + rep, nat.RUN_DIAG)
            F, T = h.loads()
            Fb, Tb = b.loads(k)
            assert np.array_equal(F, Fb) and np.array_equal(T, Tb)
            assert F.shape == (len(parts[k]), 3)
            d, db = h.diag(), b.diag(k)
            assert d.max_force == db.max_force and d.max_torque == db.max_torque
            assert tuple(d.force_sum) == tuple(db.force_sum)
            # the IMB sums come from the window reductions, grouped differently in a batch
            scale = max(np.abs(F).sum(), 1e-300)
            assert abs(d.momentum_residual - db.momentum_residual) <= 1e-12 * scale
            h.close()
        b.step(1, nat.RUN_DIAG)
    b.close()


def test_dropin_reporting_graph_follows_particle_updates():
    """A collide_stream_psc() call replays a captured CUDA graph of the whole reporting step once its
    launches repeat (one graph per buffer parity: eager, eager, capture, capture, replay, ...).  Ten
    calls of a non-static solver with the particles moved and spun between calls (geometry and solid
    velocity rebuilt outside the graph, read by it), then a particle removed (new launch arguments: run
    eagerly and captured again), stay bit-identical to the oracle."""
    from particuology_hydraulic_penalty_b200 import SparsePscD3Q19

    w = _window(20, "preloaded", 11)
    parts = w.particles.copy()
    parts[:, 4] = 1e-3
    parts[:, 9] = 2e-4
    g = SparsePscD3Q19(w.n, parts.copy(), tau=0.8, subsamples=2, body_force_z=2e-6, static_geometry=False)
    o = orc.OracleSolver(w.n, parts.copy(), tau=0.8, subsamples=2, body_force_z=2e-6, static_geometry=False)
    shape = (w.n,) * 3

    def run(arr, calls, shift0):
        for step in range(calls):
            moved = arr.copy()
            moved[:, 0] += 0.21 * (shift0 + step)
            moved[:, 1] -= 0.13 * (shift0 + step)
            g.particles = moved
            o.particles = moved.copy()
            dg = g.collide_stream_psc()
            do = o.collide_stream_psc()
            assert abs(dg["max_force"] - do["max_force"]) <= 1e-12 * do["max_force"]
            assert abs(dg["mean_uz"] - do["mean_uz"]) <= 1e-12 * max(abs(do["mean_uz"]), np.abs(o.uz).max())
        assert np.array_equal(g.f.reshape((19, *shape)), o.f)
        assert np.array_equal(g.solid, o.solid)
        fe, te = golden_io.load_errors(g.hydro_forces, g.hydro_torques, o.hydro_forces, o.hydro_torques, arr[:, 3])
        assert fe <= 1e-12 and te <= 1e-12

    run(parts, 10, 0)
    run(parts[:-1], 5, 10)


def test_batch_set_particles_all_rejects_a_window_and_keeps_every_state():
    """A non-finite particle state in one window: psc_batch_set_particles_all fails and no window takes
    a new state, including the windows before the rejected one (one of them also changes its particle
    count, which moves every later window's slot in the shared upload buffer), and a rejected set
    that would need a larger upload buffer leaves the windows on the buffer they read.  Fields and
    torques match a batch that was given only the accepted states."""
    from particuology_hydraulic_penalty_b200 import _native as nat

    wins = _three()
    a = _batch(wins)
    b = _batch(wins)
    new = [w.particles.copy() for w in wins]
    for m in new:
        m[:, 0] += 0.25
    new[0] = new[0][:-1]  # one particle fewer in window 0
    bad = [new[0], new[1].copy(), new[2]]
    bad[1][0, 2] = np.nan
    with pytest.raises(nat.PscError):
        b.set_particles_all(bad)
    a.step(2, nat.RUN_DIAG)
    b.step(2, nat.RUN_DIAG)
    for k in range(len(wins)):
        assert np.array_equal(a.loads(k)[1], b.loads(k)[1])
        assert np.array_equal(a.field(k, nat.FIELD_F), b.field(k, nat.FIELD_F))
    # and a valid set afterwards is taken by every window
    b.set_particles_all(new)
    for k, m in enumerate(new):
        a.set_particles(k, m)
    a.step(2, nat.RUN_DIAG)
    b.step(2, nat.RUN_DIAG)
    for k in range(len(wins)):
        assert np.array_equal(a.loads(k)[1], b.loads(k)[1])
        assert np.array_equal(a.field(k, nat.FIELD_F), b.field(k, nat.FIELD_F))
    # a rejected set that needs a larger upload buffer than the last one: the windows keep reading
    # the states uploaded before (the buffer is not replaced under them)
    grown = [new[0], np.concatenate([new[1]] * 4), new[2]]
    grown[1][-1, 0] = np.inf
    with pytest.raises(nat.PscError):
        b.set_particles_all(grown)
    a.step(2, nat.RUN_DIAG)
    b.step(2, nat.RUN_DIAG)
    for k in range(len(wins)):
        assert np.array_equal(a.loads(k)[1], b.loads(k)[1])
        assert np.array_equal(a.field(k, nat.FIELD_F), b.field(k, nat.FIELD_F))

def test_batch_reporting_steps_after_freezing():
    """Converged windows freeze (their state and loads stay as at convergence) and drop out of the
    all-windows loads launch; a reporting step afterwards gives the windows still running exactly
    the loads of a batch that never froze anything, run for the same number of steps."""
    from particuology_hydraulic_penalty_b200 import _native as nat

    wins = _three()
    b = _batch(wins, graph_steps=10)
    st = b.converge(tol=3e-3, check_every=20, max_steps=22)
    conv = [bool(st[k].converged) for k in range(len(wins))]
    done = [int(st[k].steps_done) for k in range(len(wins))]
    assert any(conv) and not all(conv), (conv, done)
    total = max(done)
    st2 = b.step(2, nat.RUN_DIAG)
    ref = _batch(wins, graph_steps=10)
    ref.step(total + 2, nat.RUN_DIAG)
    for k in range(len(wins)):
        if conv[k]:
            assert st2[k].steps_done == 0
            continue
        Fa, Ta = b.loads(k)
        Fr, Tr = ref.loads(k)
        assert np.array_equal(Fa, Fr) and np.array_equal(Ta, Tr)
        assert np.array_equal(b.field(k, nat.FIELD_F), ref.field(k, nat.FIELD_F))


def test_errors_are_kept_per_handle():
    """A failing call leaves its message on its own handle (and on the calling thread); other handles
    keep theirs."""
    import ctypes

    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.handle import BatchHandle, SolverHandle, make_config

    lib = nat.load()
    cfg = make_config((16, 16, 16), tau=0.8, force=(0.0, 0.0, 1e-6), subsamples=2, store=nat.STORE_F32)
    a, b = SolverHandle(cfg), SolverHandle(cfg)
    st = nat.PscStatus()
    assert lib.psc_solver_last_error(b._h) == b""
    assert lib.psc_step(a._h, -1, 0, ctypes.byref(st)) == nat.PSC_E_INVALID
    assert b"negative step count" in lib.psc_solver_last_error(a._h)
    assert b"negative step count" in lib.psc_last_error()
    assert lib.psc_solver_last_error(b._h) == b""
    assert lib.psc_converge(b._h, 0, 1e-8, 1, 1, 0, ctypes.byref(st)) == nat.PSC_E_INVALID
    assert b"max_steps" in lib.psc_solver_last_error(b._h)
    assert b"negative step count" in lib.psc_solver_last_error(a._h)
    a.step(1, nat.RUN_DIAG)  # a successful call keeps the last failure's message
    assert b"negative step count" in lib.psc_solver_last_error(a._h)
    bh = BatchHandle([cfg, cfg], graph_steps=0)
    assert lib.psc_batch_step(bh._h, -1, 0, None) == nat.PSC_E_INVALID
    assert b"negative step count" in lib.psc_batch_last_error(bh._h)
    for h in (a, b, bh):
        h.close()
