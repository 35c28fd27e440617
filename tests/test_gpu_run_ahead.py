"""Reporting steps of a batch with the next step run ahead.

A reporting step needs the post-stream moment sums of its state.  The next
step's pull computes exactly those sums (the same per-cell arithmetic and tile
order in the pair kernel), so when the step inputs have not changed since the
previous reporting call, psc_batch_step runs that next step into the other
buffer and IMB field instead of a reduction-only pass, and the next call takes
it as its first step if its inputs are still the same.  A call with
PSC_RUN_FIELDS always takes the reduction pass, so two batches of the same
windows, one stepped with PSC_RUN_DIAG and one with PSC_RUN_DIAG |
PSC_RUN_FIELDS, must report the same diagnostics, loads, populations and IMB
fields bit for bit, through every way a call can use or drop the step run
ahead: repeated reporting calls, moved particles (a rebuilt geometry), plain
steps after a reporting call, and a convergence loop.  The single-window
handle (one psc_step(h, 1, PSC_RUN_DIAG) per collide_stream_psc() call) does
the same in every kernel it runs: the exact FP64 kernel, the FP32 pair kernel
and the one-cell kernel.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIAG_FIELDS = ("solid_volume_lu", "mean_uz", "momentum_residual", "max_force", "max_torque", "mean_u",
               "superficial_u", "fluid_volume_lu", "imb_sum", "force_sum", "permeability", "nonfinite_cells")


def _pair():
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.handle import BatchHandle, make_config

    wins = [wgen.make_window(24, "skeleton", 1), wgen.make_window(32, "passive", 2),
            wgen.make_window(40, "preloaded", 3)]
    cfgs = [make_config((w.n,) * 3, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4, store=nat.STORE_F32,
                        static_geometry=False) for w in wins]
    ahead = BatchHandle(cfgs, graph_steps=4)
    plain = BatchHandle(cfgs, graph_steps=4)
    return nat, wins, ahead, plain


def _diag_tuple(d):
    out = []
    for name in DIAG_FIELDS:
        v = getattr(d, name)
        out.extend(list(v) if hasattr(v, "__len__") else [v])
    return np.array(out)


def _same(nat, a, b, nwin, loads=True):
    for k in range(nwin):
        assert np.array_equal(_diag_tuple(a.diag(k)), _diag_tuple(b.diag(k)), equal_nan=True)
        if loads:
            Fa, Ta = a.loads(k)
            Fb, Tb = b.loads(k)
            assert np.abs(Fa).sum() > 0.0
            assert np.array_equal(Fa, Fb) and np.array_equal(Ta, Tb)


def _report(nat, h, arrays, fields):
    h.set_particles_all(arrays)
    h.step(1, nat.RUN_DIAG | (nat.RUN_FIELDS if fields else 0))


def test_reporting_calls_run_ahead_equal_reduction_pass():
    nat, wins, ahead, plain = _pair()
    arrays = [w.particles for w in wins]
    for call in range(6):
        _report(nat, ahead, arrays, False)
        _report(nat, plain, arrays, True)
        _same(nat, ahead, plain, len(wins))
    for k in range(len(wins)):
        for which in (nat.FIELD_F, nat.FIELD_IMB_X, nat.FIELD_IMB_Z, nat.FIELD_UZ):
            assert np.array_equal(ahead.field(k, which), plain.field(k, which))
    ahead.close()
    plain.close()


def test_moved_particles_drop_the_step_run_ahead():
    nat, wins, ahead, plain = _pair()
    arrays = [w.particles for w in wins]
    for _ in range(3):
        _report(nat, ahead, arrays, False)
        _report(nat, plain, arrays, True)
    moved = [a.copy() for a in arrays]
    moved[1][:, 0] += 0.37  # window 1's geometry changes; the step run ahead used the old one
    for _ in range(3):
        _report(nat, ahead, moved, False)
        _report(nat, plain, moved, True)
        _same(nat, ahead, plain, len(wins))
    for k in range(len(wins)):
        assert np.array_equal(ahead.field(k, nat.FIELD_F), plain.field(k, nat.FIELD_F))
    ahead.close()
    plain.close()


def test_plain_steps_and_convergence_after_a_step_run_ahead():
    nat, wins, ahead, plain = _pair()
    arrays = [w.particles for w in wins]
    for _ in range(2):
        _report(nat, ahead, arrays, False)
        _report(nat, plain, arrays, True)
    # plain steps take the step run ahead as their first; the IMB field stays the reporting step's
    for h in (ahead, plain):
        h.step(5)
    for k in range(len(wins)):
        for which in (nat.FIELD_F, nat.FIELD_IMB_Y):
            assert np.array_equal(ahead.field(k, which), plain.field(k, which))
    for _ in range(3):
        _report(nat, ahead, arrays, False)
        _report(nat, plain, arrays, True)
        _same(nat, ahead, plain, len(wins))
    # a multi-step reporting call after a step run ahead
    for h, f in ((ahead, 0), (plain, nat.RUN_FIELDS)):
        h.step(4, nat.RUN_DIAG | f)
    _same(nat, ahead, plain, len(wins))
    # the convergence loop drops it
    sa = ahead.converge(tol=1e-3, check_every=10, max_steps=60, freeze=False)
    sp = plain.converge(tol=1e-3, check_every=10, max_steps=60, freeze=False)
    for k in range(len(wins)):
        assert sa[k].steps_done == sp[k].steps_done
        assert np.array_equal(ahead.field(k, nat.FIELD_F), plain.field(k, nat.FIELD_F))
    _report(nat, ahead, arrays, False)
    _report(nat, plain, arrays, True)
    _same(nat, ahead, plain, len(wins))
    ahead.close()
    plain.close()


# ---- single-window handle (the drop-in's collide_stream_psc() calls) -------------------------

def _solo_pair(store_name, n, static=True):
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.handle import SolverHandle, make_config

    w = wgen.make_window(n, "preloaded", 11)
    cfg = make_config((n,) * 3, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4, store=getattr(nat, store_name),
                      static_geometry=static)
    a, b = SolverHandle(cfg), SolverHandle(cfg)
    return nat, w, a, b


def _solo_same(nat, a, b):
    assert np.array_equal(_diag_tuple(a.step_diag), _diag_tuple(b.step_diag), equal_nan=True)
    Fa, Ta = a.loads()
    Fb, Tb = b.loads()
    assert np.abs(Fa).sum() > 0.0
    assert np.array_equal(Fa, Fb) and np.array_equal(Ta, Tb)


def _solo_report(nat, h, particles, fields):
    h.set_particles(particles)
    h.step_diag = h.step(1, nat.RUN_DIAG | (nat.RUN_FIELDS if fields else 0)).diag


@pytest.mark.parametrize("store_name,n", [("STORE_F64_EXACT", 24), ("STORE_F32", 32), ("STORE_F32", 27)])
def test_solver_reporting_calls_run_ahead_equal_reduction_pass(store_name, n):
    """FP64-exact (its own kernel), FP32 pair kernel (even nz) and FP32 one-cell kernel (odd nz)."""
    nat, w, a, b = _solo_pair(store_name, n)
    for _ in range(6):  # eager, captured and replayed calls of every kind
        _solo_report(nat, a, w.particles, False)
        _solo_report(nat, b, w.particles, True)
        _solo_same(nat, a, b)
    for which in (nat.FIELD_F, nat.FIELD_IMB_X, nat.FIELD_IMB_Z, nat.FIELD_UZ):
        assert np.array_equal(a.field(which), b.field(which))
    # a loads call on the current IMB field repeats the reporting call's loads
    Fa, Ta = a.loads()
    a.accumulate_loads()
    Fc, Tc = a.loads()
    assert np.array_equal(Fa, Fc) and np.array_equal(Ta, Tc)
    a.close()
    b.close()


def test_solver_run_ahead_dropped_by_other_calls():
    nat, w, a, b = _solo_pair("STORE_F32", 32, static=False)
    for _ in range(3):
        _solo_report(nat, a, w.particles, False)
        _solo_report(nat, b, w.particles, True)
    moved = w.particles.copy()
    moved[:, 2] += 0.29  # a rebuilt geometry
    for _ in range(3):
        _solo_report(nat, a, moved, False)
        _solo_report(nat, b, moved, True)
        _solo_same(nat, a, b)
    for h in (a, b):
        h.step(3)  # plain steps overwrite the other buffer
    _solo_report(nat, a, moved, False)
    _solo_report(nat, b, moved, True)
    _solo_same(nat, a, b)
    _solo_report(nat, a, moved, False)
    _solo_report(nat, b, moved, True)
    f = a.field(nat.FIELD_F)
    for h in (a, b):
        h.set_populations(f)  # a new state
    for _ in range(2):
        _solo_report(nat, a, moved, False)
        _solo_report(nat, b, moved, True)
        _solo_same(nat, a, b)
    assert np.array_equal(a.field(nat.FIELD_F), b.field(nat.FIELD_F))
    a.close()
    b.close()
