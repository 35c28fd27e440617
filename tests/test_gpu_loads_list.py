"""Particle loads through the loads list: the first call on a geometry and the later ones agree
bit for bit.

The first loads call on a geometry builds its list -- the bbox entries with a
non-zero count and their owner weights alpha_p / max(alpha_sum, 1e-14)
(psc3d.py:386), dealt to the lanes of each warp -- and reduces from it; later
calls on the same geometry reduce from the list without building it.  Two runs
reach the same state: one takes two steps in one call (its only loads call
builds the list), the other takes two one-step calls (its second loads call
reuses the list).  Forces, torques and load diagnostics must agree exactly, for
one window and for a batch, in FP32 and in the exact FP64 mode.  A geometry
rebuilt for moved particles must not reuse the old list.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _windows():
    from particuology_hydraulic_penalty_b200 import windows as wgen

    return [wgen.make_window(48, "preloaded", 7), wgen.make_window(64, "passive", 8)]


@pytest.mark.parametrize("store_name", ["STORE_F32", "STORE_F64_EXACT"])
def test_solver_list_loads_bitwise(store_name):
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.handle import SolverHandle, make_config

    w = _windows()[0]
    store = getattr(nat, store_name)
    cfg = make_config((w.n,) * 3, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4, store=store)
    a = SolverHandle(cfg)
    a.set_particles(w.particles)
    da = a.step(2, nat.RUN_DIAG).diag
    Fa, Ta = a.loads()
    b = SolverHandle(cfg)
    b.set_particles(w.particles)
    b.step(1, nat.RUN_DIAG)
    db = b.step(1, nat.RUN_DIAG).diag
    Fb, Tb = b.loads()
    assert np.abs(Fa).sum() > 0.0
    assert np.array_equal(Fa, Fb)
    assert np.array_equal(Ta, Tb)
    assert da.momentum_residual == db.momentum_residual
    assert da.max_force == db.max_force and da.max_torque == db.max_torque
    # a loads call on the current IMB field of the same geometry (list path) repeats them
    b.accumulate_loads()
    Fc, Tc = b.loads()
    assert np.array_equal(Fb, Fc) and np.array_equal(Tb, Tc)
    a.close()
    b.close()


def test_batch_list_loads_bitwise():
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.handle import BatchHandle, make_config

    wins = _windows()
    cfgs = [make_config((w.n,) * 3, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4, store=nat.STORE_F32)
            for w in wins]
    a = BatchHandle(cfgs, graph_steps=0)
    b = BatchHandle(cfgs, graph_steps=0)
    for k, w in enumerate(wins):
        a.set_particles(k, w.particles)
        b.set_particles(k, w.particles)
    a.step(2, nat.RUN_DIAG)
    b.step(1, nat.RUN_DIAG)
    b.step(1, nat.RUN_DIAG)
    for k in range(len(wins)):
        Fa, Ta = a.loads(k)
        Fb, Tb = b.loads(k)
        assert np.abs(Fa).sum() > 0.0
        assert np.array_equal(Fa, Fb) and np.array_equal(Ta, Tb)
        assert a.diag(k).momentum_residual == b.diag(k).momentum_residual
    a.close()
    b.close()


def test_rebuilt_geometry_drops_its_loads_list():
    """Dynamic geometry: moving the particles after the loads list of the first geometry was written
    rebuilds the geometry.  The next step's loads equal those of a fresh solver that starts from the
    same populations with the moved particles (its first loads call reduces the whole boxes)."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.handle import SolverHandle, make_config

    w = _windows()[0]
    cfg = make_config((w.n,) * 3, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4, store=nat.STORE_F64_EXACT,
                      static_geometry=False)
    a = SolverHandle(cfg)
    a.set_particles(w.particles)
    a.step(1, nat.RUN_DIAG)
    a.step(1, nat.RUN_DIAG)  # loads list of the first geometry written and used
    moved = w.particles.copy()
    moved[:, 0] += 0.37  # every sphere shifts along x: a different geometry
    a.set_particles(moved)
    f = a.field(nat.FIELD_F)
    a.step(1, nat.RUN_DIAG)
    Fa, Ta = a.loads()
    b = SolverHandle(cfg)
    b.set_particles(moved)
    b.set_populations(f)
    b.step(1, nat.RUN_DIAG)  # first loads call on this geometry: whole boxes
    Fb, Tb = b.loads()
    assert np.array_equal(Fa, Fb) and np.array_equal(Ta, Tb)
    a.close()
    b.close()


def _device_status():
    import ctypes

    from particuology_hydraulic_penalty_b200 import _native as nat

    v = ctypes.c_int(0)
    nat.call("psc_device_status", ctypes.byref(v), 1)
    return v.value


def test_chunk_rows_with_many_chunks_per_block():
    """The load-chunk kernels write a chunk's row from the warp that finishes the chunk last, through
    a ring of four partial-sum slots per block; a warp may run ahead of the others by up to four
    chunks.  On the 24 windows of the benchmark batch (about 15 000 chunks for 2368 blocks) every
    block reuses its slots, in the first step (list built, then reduced) and in the second (list
    reused).  Each window's forces and torques equal those of the window run alone, where a block
    holds far fewer chunks, bit for bit, and no kernel gave up a wait."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.handle import BatchHandle, SolverHandle, make_config

    _device_status()
    wins = wgen.batched_windows(24, seed0=0)
    cfgs = [make_config((w.n,) * 3, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4, store=nat.STORE_F32)
            for w in wins]
    b = BatchHandle(cfgs, graph_steps=0)
    b.set_particles_all([w.particles for w in wins])
    b.step(1, nat.RUN_DIAG)
    whole = [b.loads(k) for k in range(len(wins))]
    b.step(1, nat.RUN_DIAG)
    listed = [b.loads(k) for k in range(len(wins))]
    assert _device_status() == 0
    for k in (0, 1, 5, 11, 17, 23):
        s = SolverHandle(cfgs[k])
        s.set_particles(wins[k].particles)
        s.step(1, nat.RUN_DIAG)
        F1, T1 = s.loads()
        s.step(1, nat.RUN_DIAG)
        F2, T2 = s.loads()
        s.close()
        assert np.abs(F1).sum() > 0.0
        assert np.array_equal(whole[k][0], F1) and np.array_equal(whole[k][1], T1)
        assert np.array_equal(listed[k][0], F2) and np.array_equal(listed[k][1], T2)
    assert _device_status() == 0
    b.close()
