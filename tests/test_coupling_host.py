"""Coupling helpers against the reference's formulas (CPU)."""

import math

import numpy as np

from particuology_hydraulic_penalty_b200 import coupling


def test_si_scaling_formulas():
    s = coupling.apply_si_scaling(64, 0.8)
    rho = 2.0e5 / (2077.1 * 773.15)
    nu = 3.7e-5 / rho
    nu_lu = (0.8 - 0.5) / 3.0
    dx = 0.009 / 64
    dt = nu_lu * dx * dx / nu
    assert math.isclose(s["dt_s"], dt, rel_tol=1e-15)
    assert math.isclose(s["force_scale_N_per_lu"], rho * dx ** 4 / dt ** 2, rel_tol=1e-15)
    assert math.isclose(s["torque_scale_Nm_per_lu"], rho * dx ** 5 / dt ** 2, rel_tol=1e-15)
    assert math.isclose(s["velocity_lu_per_m_s"], dt / dx, rel_tol=1e-15)


def test_particles_from_state():
    x = np.array([[0.0045, 0.001, 0.002]])
    p = coupling.psc_particles_from_state(x, [[1e-3, 0, 0]], [[0, 2.0, 0]], [0.0003], 64, 10.0, 0.5)
    assert np.allclose(p[0, :4], [32.0, 64 * 0.001 / 0.009, 64 * 0.002 / 0.009, 64 * 0.0003 / 0.009])
    assert np.allclose(p[0, 4:], [1e-2, 0, 0, 0, 1.0, 0])


class _FakeSolver:
    """Stands in for the GPU solver: mean_uz approaches a limit geometrically."""

    def __init__(self):
        self.k = 0
        self.uz = np.zeros((2, 2, 2))

    def collide_stream_psc(self):
        self.k += 1
        return {"mean_uz": 1.0 - 0.5 ** self.k}


def test_converge_semantics():
    it, res, ok, diag = coupling.lbm_converge(_FakeSolver(), residual_tol=1e-3, min_steps=3, max_steps=100)
    # residual_k = 2^-k / (1 - 2^-k) falls below 1e-3 at k = 10
    assert ok and it == 10 and res < 1e-3
    it, res, ok, _ = coupling.lbm_converge(_FakeSolver(), residual_tol=1e-12, min_steps=1, max_steps=5)
    assert not ok and it == 5
    steps, res, ok, diag = coupling.lbm_transient_advance(_FakeSolver(), 4)
    assert steps == 4 and ok and math.isclose(diag["mean_uz"], 1 - 0.5 ** 4)


def test_validation_profiles_and_steady_rule():
    """The validation campaign's profile grids are those the golden rows were made with, and the
    steady-state rule (validation/run_precision_validation.py:148-158, :223-233) on known series."""
    import json
    from pathlib import Path

    from particuology_hydraulic_penalty_b200 import validation as val

    gold = json.loads((Path(__file__).resolve().parent / "golden" / "validation_quick.json").read_text())
    prof = val.PROFILES["quick"]
    runs = [prof.settling, *prof.hasimoto, *prof.permeability]
    assert [(r["n"], r["radius_lu"], r["subsamples"]) for r in gold["rows"]] == \
        [(g.n, g.radius, prof.subsamples) for g in runs]
    assert [len(val.PROFILES[p].hasimoto) for p in ("quick", "standard", "high")] == [2, 3, 3]
    flat = [1.0] * 8
    assert val.steady_metrics(flat) == (0.0, 0.0)
    run = val.GridRun(20, 2.5, 100, 800, 20)
    assert not val.should_stop(99, run, flat, 1e-2)          # before min_steps
    assert not val.should_stop(200, run, flat[:7], 1e-2)     # fewer than 8 samples
    assert val.should_stop(200, run, flat, 1e-2)
    assert not val.should_stop(200, run, flat, 1e-2, extra_check=lambda: False)
    rising = [1.0 + 0.01 * k for k in range(8)]
    std_rel, drift_rel = val.steady_metrics(rising)
    assert drift_rel > 1e-2 and not val.should_stop(200, run, rising, 1e-2)
    assert abs(val.hasimoto_factor(2.5, 20.0) - 1.0 / (1.0 - 2.837297 * 0.125 + 4.19 * 0.125 ** 3
                                                        - 27.4 * 0.125 ** 6)) < 1e-15
