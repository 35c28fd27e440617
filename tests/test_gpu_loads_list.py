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


def test_list_layout_is_the_documented_one():
    """psc_particle_loads with the three list arrays and list_ready = 0 builds the list the header
    documents (include/psc_b200.h, psc_geometry): warp w of chunk c owns the entries 32w + l + 256j,
    numbers its non-zero ones in that order, and entry number n sits in slot
    c * chunk_entries + (n / 32) * 256 + 32w + n % 32 with the owner weight
    (count / S^3) / max(alpha_sum, 1e-14) and the packed bbox-local cell; load_n counts each
    thread's slots.  Rebuilt here from the geometry's own counts and alpha sums, slot by slot."""
    import ctypes

    import torch

    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.engine import DeviceGeometry, LatticeWindow, stream_handle, vp

    dev = torch.device("cuda", 0)
    n, S = 32, 3
    shape = (n, n, n)
    w = wgen.make_window(n, "preloaded", 5)
    with torch.cuda.device(dev):
        geo = DeviceGeometry(shape, S, dev, want_level=True)
        geo.set_particles(w.particles)
        geo.rebuild()
        win = LatticeWindow(shape, 0.8, (1e-6, 0.0, 0.0), S, nat.STORE_F32, None, dev)
        win.bind_geometry(geo)
        win.step(nat.STEP_IMB | nat.STEP_REDUCE)
        win.reduce(win.red)
        g = geo.struct()
        CE, C, P = int(g.chunk_entries), int(g.capacity_chunks), int(g.nparticles)
        lw = torch.full((C * CE,), float("nan"), dtype=torch.float64, device=dev)
        labk = torch.zeros(C * CE, dtype=torch.int32, device=dev)
        ln = torch.full((C * 256,), 255, dtype=torch.uint8, device=dev)
        g.load_w, g.load_abk, g.load_n, g.list_ready = lw.data_ptr(), labk.data_ptr(), ln.data_ptr(), 0
        F = torch.zeros((P, 3), dtype=torch.float64, device=dev)
        T = torch.zeros((P, 3), dtype=torch.float64, device=dev)
        D = torch.zeros(nat.NDIAG, dtype=torch.float64, device=dev)
        nat.call("psc_particle_loads", ctypes.byref(g), 1, vp(win.imb), vp(geo.chunk_partials),
                 vp(win.red[nat.RED_IMBX:]), vp(F), vp(T), vp(D), stream_handle(dev))
        torch.cuda.synchronize()
    cnt = geo.ent_cnt.cpu().numpy().view(np.uint16)
    alpha = geo.alpha_sum.cpu().numpy()
    bbox = geo.bbox.cpu().numpy().reshape(-1, 6)
    ent_off = geo.ent_off.cpu().numpy()
    chunk_off = geo.chunk_off.cpu().numpy()
    lw_h, labk_h, ln_h = lw.cpu().numpy(), labk.cpu().numpy().view(np.uint32), ln.cpu().numpy()
    S3 = np.float64(S ** 3)
    listed = 0
    for p in range(P):
        x0, y0, z0, _, ey, ez = (int(v) for v in bbox[p])
        for c in range(int(chunk_off[p]), int(chunk_off[p + 1])):
            e0 = int(ent_off[p]) + (c - int(chunk_off[p])) * CE
            e1 = min(e0 + CE, int(ent_off[p + 1]))
            for warp in range(8):
                mine = [e0 + 32 * warp + lane + 256 * j for j in range(CE // 256) for lane in range(32)]
                nonzero = [e for e in mine if e < e1 and cnt[e] != 0]
                for num, e in enumerate(nonzero):
                    local = e - int(ent_off[p])
                    a, rem = divmod(local, ey * ez)
                    b, k = divmod(rem, ez)
                    cell = ((x0 + a) * n + (y0 + b)) * n + (z0 + k)
                    ow = (np.float64(cnt[e]) / S3) / max(alpha[cell], 1e-14)
                    slot = c * CE + (num >> 5) * 256 + 32 * warp + (num & 31)
                    assert lw_h[slot] == ow and labk_h[slot] == (a | (b << 11) | (k << 22))
                    listed += 1
                for lane in range(32):
                    want = (len(nonzero) - lane + 31) // 32 if len(nonzero) > lane else 0
                    assert ln_h[c * 256 + 32 * warp + lane] == want
    assert listed > 1000
    assert np.abs(F.cpu().numpy()).sum() > 0.0
