"""The CPU oracle reproduces the reference kernel's own outputs (golden fixtures).

Fields are compared with ``==`` (bit-exact up to the sign of zero); force and
torque sums, whose NumPy pairwise order differs between the reference's dense
and sparse classes, to 1e-13 relative in vector norm.
"""

import numpy as np
import pytest

from oracle import psc_oracle as orc
from tests import golden_io

CASES = golden_io.names()


def run_oracle(data):
    m = data["meta"]
    s = orc.OracleSolver(m["n"], data["particles"], tau=m["tau"], subsamples=m["subsamples"],
                         body_force_z=m["force_z"], static_geometry=m["static"])
    diags, first = [], None
    for step in range(m["steps"]):
        d = s.collide_stream_psc()
        diags.append([d["solid_volume_lu"], d["mean_uz"], d["momentum_residual"], d["max_force"],
                      d["max_torque"]])
        if step == 0:
            first = (s.f.copy(), s.hydro_forces.copy(), s.hydro_torques.copy())
    return s, np.asarray(diags), first


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(name):
    data = golden_io.load(name)
    s, diags, first = run_oracle(data)
    assert np.array_equal(s.solid, data["solid"])
    for key in ("rho", "ux", "uy", "uz"):
        assert np.array_equal(getattr(s, key), data[key]), key
    assert np.array_equal(s.imb, data["imb"])
    assert np.array_equal(s.f, data["f"])
    if "f_step1" in data:
        assert np.array_equal(first[0], data["f_step1"])
    radii = data["particles"][:, 3]
    fe, te = golden_io.load_errors(s.hydro_forces, s.hydro_torques, data["hydro_forces"],
                                   data["hydro_torques"], radii)
    assert fe <= 1e-13 and te <= 1e-13, (fe, te)
    fe1, te1 = golden_io.load_errors(first[1], first[2], data["hydro_forces_step1"],
                                     data["hydro_torques_step1"], radii)
    assert fe1 <= 1e-13 and te1 <= 1e-13, (fe1, te1)
    # solid volume and mean uz come from identical fields and identical numpy sums
    assert np.array_equal(diags[:, 0], data["diags"][:, 0])
    assert np.array_equal(diags[:, 1], data["diags"][:, 1])
    # the momentum residual is a round-off quantity: compare against the force scale
    scale = max(1e-300, float(np.abs(data["hydro_forces"]).sum()))
    assert abs(diags[-1, 2] - data["diags"][-1, 2]) <= 1e-12 * scale + 1e-300
    if data["meta"]["kind"] == "sparse":
        ids, vals = golden_io.sparse_lists(data)
        assert len(ids) == len(s.geo.node_ids)
        for a, b, va, vb in zip(s.geo.node_ids, ids, s.geo.alpha_vals, vals):
            assert np.array_equal(a, b)
            assert np.array_equal(va, vb)
        assert np.array_equal(s.geo.alpha_sum_flat, data["alpha_sum_flat"])
    else:
        assert np.array_equal(orc.dense_alpha(s.geo), data["alpha_p"])


def test_reference_smoke_assertions_hold_on_oracle():
    """The reference's own smoke test (tests/test_psc3d_smoke.py:6-23) on the oracle."""
    s = orc.OracleSolver(12, np.array([[6.0, 6.0, 6.0, 2.0] + [0.0] * 6]),
                         tau=0.72, subsamples=2, body_force_z=1.0e-7, static_geometry=True)
    d = s.collide_stream_psc()
    assert 0.0 < s.solid.mean() < 1.0
    assert np.isfinite(s.f).all()
    assert np.isfinite(s.hydro_forces).all()
    assert np.isfinite(d["momentum_residual"])


def test_trt_extension_reduces_to_bgk():
    """The oracle's TRT extension with tau_minus = tau equals the reference collision."""
    rng = np.random.default_rng(2)
    shp = (5, 5, 5)
    f = orc.equilibrium(1 + rng.normal(0, 1e-3, shp), *rng.normal(0, 1e-3, (3,) + shp))
    f = f + rng.normal(0, 1e-6, f.shape) * orc.W[:, None, None, None]
    solid = rng.choice([0.0, 0.25, 1.0], size=shp)
    F = (1e-5, 0.0, 2e-6)
    post, _ = orc.collide(f, solid, None, 0.8, F)
    trt = orc.collide_trt_deviation(f - orc.W[:, None, None, None], solid, 0.8, 0.8, F)
    assert np.abs(trt + orc.W[:, None, None, None] - post).max() <= 2e-16
