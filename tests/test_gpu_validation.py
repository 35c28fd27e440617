"""The reference's precision-validation campaign on the GPU, quick profile, against the summary rows the
reference itself produced (tests/golden/validation_quick.json, made by make_validation_golden.py from
validation/run_precision_validation.py).

The drop-in runs the reference's arithmetic (fp64-exact), so every case must stop at the same step
with the same steady-state and force-balance verdicts, and every measured figure must agree to
round-off (the fluid sums are taken in another order on the GPU; the settling sphere integrates the
forces, which agree to 1e-12).  The verdicts of the reference's own checks (time_converged,
force_balance_pass) must be the same: at the quick profile the settling and Hasimoto cases reach
steady state (settling also balances its forces), while the fixed-array permeability case runs out of
steps before its permeability settles and fails the force balance, in the reference as here."""

import json
import math
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "validation_quick.json").read_text())
REL = 1e-9


def _close(a, b, rel=REL):
    if isinstance(b, str) or isinstance(a, str):
        return a == b
    if isinstance(b, float) and math.isnan(b):
        return isinstance(a, float) and math.isnan(a)
    return abs(float(a) - float(b)) <= rel * max(abs(float(b)), 1e-300) + 1e-300


def _check(row, ref):
    assert row["case"] == ref["case"] and row["n"] == ref["n"]
    assert row["steps"] == ref["steps"], (row["steps"], ref["steps"])
    assert row["time_converged"] == ref["time_converged"]
    assert row["force_balance_pass"] == ref["force_balance_pass"]
    for key in ("reference_value", "measured_value", "signed_relative_error", "force_ratio_tail",
                "effective_force_ratio_tail", "force_balance_relative", "re_tail", "hasimoto_factor",
                "exact_porosity", "psc_porosity", "solid_volume_relative_error"):
        assert _close(row[key], ref[key]), (key, row[key], ref[key])
    # steady-state spreads are differences of nearly equal samples: compare on the samples' scale
    for key in ("steady_std_relative", "steady_drift_relative"):
        assert abs(row[key] - ref[key]) <= 1e-9, (key, row[key], ref[key])
    # the closure residual is round-off in both
    assert row["momentum_residual_tail"] <= 1e-12 * max(1.0, abs(ref["measured_value"]))


def _ref_rows(case):
    return [r for r in GOLDEN["rows"] if r["case"] == case]


def test_settling_quick_matches_reference():
    from particuology_hydraulic_penalty_b200 import validation as val

    row = val.run_settling("quick", val.PROFILES["quick"], GOLDEN["meta"]["tau"],
                           GOLDEN["meta"]["particle_density_ratio"])
    (ref,) = _ref_rows("single_particle_settling")
    _check(row, ref)
    assert row["time_converged"] == 1 and row["force_balance_pass"] == 1


def test_hasimoto_quick_matches_reference():
    from particuology_hydraulic_penalty_b200 import validation as val

    prof = val.PROFILES["quick"]
    refs = _ref_rows("periodic_moving_sphere_hasimoto")
    assert len(refs) == len(prof.hasimoto)
    for run, ref in zip(prof.hasimoto, refs):
        row = val.run_hasimoto_case("quick", prof, run, GOLDEN["meta"]["tau"])
        _check(row, ref)
        assert row["time_converged"] == 1


def test_fixed_array_permeability_quick_matches_reference():
    from particuology_hydraulic_penalty_b200 import validation as val

    prof = val.PROFILES["quick"]
    (ref,) = _ref_rows("periodic_fixed_array_permeability")
    row = val.run_permeability_case("quick", prof, prof.permeability[0], GOLDEN["meta"]["tau"])
    _check(row, ref)
    assert row["force_balance_pass"] == ref["force_balance_pass"]


def test_profile_table_and_report(tmp_path):
    from particuology_hydraulic_penalty_b200 import validation as val

    rows = val.run_profile("quick", cases=("hasimoto",), tau=GOLDEN["meta"]["tau"], out_dir=tmp_path)
    assert len(rows) == 2
    assert (tmp_path / "precision_error_table.csv").read_text().splitlines()[0].split(",") == val.SUMMARY_FIELDS
    assert "periodic_moving_sphere_hasimoto" in (tmp_path / "precision_validation_report.md").read_text()
