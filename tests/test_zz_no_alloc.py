"""psc_particle_loads_static: particle loads for callers that cannot allocate device memory.

Some callers of this library own no device allocator -- a DEM code's coupling
hook that is handed only the IMB field and the particle arrays, or a
coupling loop that must not call cudaMalloc once it runs (an allocation
synchronises the device).  For them psc_particle_loads_static() keeps its
per-chunk partial sums in a fixed array inside the library.  This test
calls it through the C ABI, twice in a row, and compares it with
psc_particle_loads(), which takes the caller's scratch buffer.  The file is
named to be collected last.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _particles():
    rng = np.random.default_rng(42)
    P = 30
    parts = np.zeros((P, 10))
    parts[:, 0:3] = rng.uniform(-1.0, 25.0, size=(P, 3))
    parts[:, 3] = rng.uniform(1.0, 4.0, size=P)
    parts[:, 4:7] = rng.normal(0.0, 1e-4, size=(P, 3))
    return parts


def _state(store_name="STORE_F64_EXACT", particles=None):
    """Geometry and lattice of a caller that owns the device buffers (descriptor layer), two steps in.
    The exact FP64 mode keeps a float64 IMB field (imb_type 0), the FP32 mode a float32 one (1)."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.engine import DeviceGeometry, LatticeWindow

    store = getattr(nat, store_name)
    dev = torch.device("cuda", 0)
    shape = (24, 24, 24)
    with torch.cuda.device(dev):
        geo = DeviceGeometry(shape, 3, dev, want_level=store != nat.STORE_F64_EXACT)
        geo.set_particles(_particles() if particles is None else particles)
        geo.rebuild()
        win = LatticeWindow(shape, 0.8, (0.0, 0.0, 2e-6), 3, store, None, dev)
        win.bind_geometry(geo)
        geo.solid_velocity(win.ensure_us())
        win.set_moving(True)
        for _ in range(2):
            win.step(nat.STEP_IMB | nat.STEP_REDUCE)
        win.reduce(win.red)  # IMB momentum sums of the last step
    return geo, win


def _compare_two_calls(geo, win, imb_type):
    """psc_particle_loads_static twice in a row (outputs pre-filled with NaN) against
    psc_particle_loads with the caller's scratch, to round-off (the chunk sums are added in a
    different order); returns the last outputs."""
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.engine import stream_handle, vp

    dev = win.imb.device
    g = geo.struct()
    assert g.capacity_chunks <= nat.LOADS_STATIC_MAX_CHUNKS
    P = geo.P
    imb_sums = win.red[nat.RED_IMBX:]
    ref = [torch.zeros((P, 3), dtype=torch.float64, device=dev), torch.zeros((P, 3), dtype=torch.float64, device=dev),
           torch.zeros(nat.NDIAG, dtype=torch.float64, device=dev)]
    nat.call("psc_particle_loads", ctypes.byref(g), imb_type, vp(win.imb), vp(geo.chunk_partials), vp(imb_sums),
             vp(ref[0]), vp(ref[1]), vp(ref[2]), stream_handle(dev))
    lib = nat.load()
    for _ in range(2):  # the second call reuses the shared scratch left by the first
        out = [torch.full((P, 3), float("nan"), dtype=torch.float64, device=dev),
               torch.full((P, 3), float("nan"), dtype=torch.float64, device=dev),
               torch.full((nat.NDIAG,), float("nan"), dtype=torch.float64, device=dev)]
        rc = lib.psc_particle_loads_static(ctypes.byref(g), imb_type, vp(win.imb), vp(imb_sums), vp(out[0]),
                                           vp(out[1]), vp(out[2]), stream_handle(dev))
        assert rc == nat.PSC_OK, lib.psc_last_error()
        torch.cuda.synchronize()
        for a, b in zip(out, ref):
            a, b = a.cpu().numpy(), b.cpu().numpy()
            assert np.all(np.isfinite(a))
            assert np.linalg.norm(a - b) <= 1e-12 * max(np.linalg.norm(b), 1e-300)
    return out


def test_static_scratch_loads_match_caller_scratch_loads():
    from particuology_hydraulic_penalty_b200 import SparsePscD3Q19

    geo, win = _state()
    assert geo.struct().capacity_chunks > 0
    out = _compare_two_calls(geo, win, 0)
    # the forces also match what the drop-in solver reports for the same two steps
    s = SparsePscD3Q19(24, _particles(), tau=0.8, subsamples=3, body_force_z=2e-6, static_geometry=True,
                       precision="fp64-exact")
    s.collide_stream_psc()
    s.collide_stream_psc()
    assert np.linalg.norm(out[0].cpu().numpy() - s.hydro_forces) <= 1e-12 * np.linalg.norm(s.hydro_forces)


def test_static_scratch_loads_float_imb_field():
    """A float32 IMB field (the FP32 / FP16 / BF16 storage modes' imb_type 1)."""
    geo, win = _state("STORE_F32")
    assert win.imb.dtype == torch.float32
    out = _compare_two_calls(geo, win, 1)
    assert float(out[0].abs().sum()) > 0.0


def test_static_scratch_loads_without_particles():
    """No particles (no load chunks): rc is PSC_OK and the diagnostics are still written -- the
    closure residual is the IMB momentum sum alone, the force and torque maxima are 0."""
    geo, win = _state(particles=np.zeros((0, 10)))
    assert geo.P == 0
    out = _compare_two_calls(geo, win, 0)
    diag = out[2].cpu().numpy()
    assert diag[1] == 0.0 and diag[2] == 0.0


def test_static_scratch_rejects_oversized_geometry():
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.engine import stream_handle, vp

    geo, win = _state()
    g = geo.struct()
    g.capacity_chunks = nat.LOADS_STATIC_MAX_CHUNKS + 1
    lib = nat.load()
    out = torch.zeros((geo.P, 3), dtype=torch.float64, device=win.imb.device)
    diag = torch.zeros(nat.NDIAG, dtype=torch.float64, device=out.device)
    rc = lib.psc_particle_loads_static(ctypes.byref(g), 0, vp(win.imb), vp(win.red[nat.RED_IMBX:]), vp(out),
                                       vp(out), vp(diag), stream_handle(out.device))
    assert rc == nat.PSC_E_CAPACITY
    assert b"scratch holds" in lib.psc_last_error()
