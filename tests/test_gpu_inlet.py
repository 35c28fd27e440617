"""Open-x windows on the GPU (bounce-back velocity inlet at x = 0,
zero-gradient outflow at x = nx - 1; an extension of the reference): the
exact mode reproduces the oracle's extension bit for bit, the deviation modes
within their tolerances, and batched windows match solo ones."""

import numpy as np
import pytest

from oracle import psc_oracle as orc

pytestmark = pytest.mark.gpu

INLET = (1.0, (0.004, 0.0005, -0.0003))


def _window(n=16, kind="passive", seed=11):
    from particuology_hydraulic_penalty_b200 import windows as wgen

    return wgen.make_window(n, kind, seed)


def test_exact_inlet_matches_oracle_bitwise():
    from particuology_hydraulic_penalty_b200 import SparsePscD3Q19

    w = _window()
    gpu = SparsePscD3Q19(w.n, w.particles, tau=0.8, subsamples=2, body_force_z=1e-6, static_geometry=True,
                         precision="fp64-exact", inlet=INLET)
    ref = orc.OracleSolver(w.n, w.particles, tau=0.8, subsamples=2, body_force_z=1e-6, static_geometry=True,
                           inlet=INLET)
    for _ in range(8):
        dg = gpu.collide_stream_psc()
        dr = ref.collide_stream_psc()
    assert np.array_equal(gpu.solid, ref.solid)
    assert np.array_equal(gpu.f, ref.f)
    assert np.array_equal(gpu.ux, ref.ux) and np.array_equal(gpu.uz, ref.uz)
    rel = np.linalg.norm(gpu.hydro_forces - ref.hydro_forces) / np.linalg.norm(ref.hydro_forces)
    assert rel <= 1e-12
    assert abs(dg["mean_uz"] - dr["mean_uz"]) <= 1e-12 * float(np.abs(ref.ux).max())


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_deviation_inlet_close_to_oracle(precision):
    from particuology_hydraulic_penalty_b200 import SparsePscD3Q19

    w = _window(16, "skeleton", 12)
    gpu = SparsePscD3Q19(w.n, w.particles, tau=0.8, subsamples=2, body_force_z=0.0, static_geometry=True,
                         precision=precision, inlet=INLET)
    ref = orc.OracleSolver(w.n, w.particles, tau=0.8, subsamples=2, static_geometry=True, inlet=INLET)
    for _ in range(30):
        gpu.collide_stream_psc()
        ref.collide_stream_psc()
    tol = {"fp64": 1e-10, "fp32": 2e-4}[precision]
    scale = float(np.abs(ref.ux).max())
    assert np.abs(gpu.ux - ref.ux).max() <= tol * scale
    assert np.abs(gpu.uy - ref.uy).max() <= tol * scale
    assert np.abs(gpu.f - ref.f).max() <= tol * 10 * scale


def test_batched_inlet_windows_equal_solo():
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = [_window(16, "skeleton", 1), _window(24, "passive", 2)]
    specs = [WindowSpec(wins[0].n, wins[0].particles, tau=0.8, force=(0.0, 0.0, 0.0), subsamples=4, inlet=INLET),
             WindowSpec(wins[1].n, wins[1].particles, tau=0.8, force=(1e-6, 0.0, 0.0), subsamples=4)]
    b = PscBatch(specs, precision="fp32", graph_steps=4)
    b.run(13)
    for k, spec in enumerate(specs):
        solo = PscBatch([spec], precision="fp32", graph_steps=0)
        solo.run(13)
        assert np.array_equal(solo.velocity_field(0), b.velocity_field(k))


def test_handle_post_stream_f_of_open_window():
    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.engine import store_mode
    from particuology_hydraulic_penalty_b200.handle import SolverHandle, make_config

    w = _window(12, "preloaded", 4)
    cfg = make_config((w.n,) * 3, tau=0.9, force=(0.0, 0.0, 0.0), subsamples=2, store=store_mode("fp64-exact"),
                      inlet=INLET)
    h = SolverHandle(cfg)
    h.set_particles(w.particles)
    h.step(5, nat.RUN_DIAG)
    ref = orc.OracleSolver(w.n, w.particles, tau=0.9, subsamples=2, static_geometry=True, inlet=INLET)
    for _ in range(5):
        ref.collide_stream_psc()
    assert np.array_equal(h.field(nat.FIELD_F).reshape(ref.f.shape), ref.f)
