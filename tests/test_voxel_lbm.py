"""Voxel bounce-back path: oracle pinned to the reference (CPU), GPU bit-exact to the fixtures."""

import numpy as np
import pytest

from oracle import voxel_oracle as vo
from tests import golden_io

VOXEL = golden_io.voxel_names()


@pytest.mark.parametrize("name", VOXEL)
def test_voxel_oracle_matches_reference(name):
    d = golden_io.load(name)
    m = d["meta"]
    solid, dx = vo.voxelize(d["points"], d["center"], d["size"], m["radius"], m["n"])
    assert np.array_equal(solid, d["solid"]) and np.array_equal(dx, d["dx"])
    res = vo.run_lbm(solid, m["tau"], m["force_z"], m["steps"], return_fields=True)
    for k in ("ux", "uy", "uz"):
        assert np.array_equal(res[k], d[k]), k
    got = [res["mean_uz_fluid"], res["superficial_uz"], res["max_uz"], res["permeability_lu"], res["porosity_voxel"]]
    assert np.array_equal(np.asarray(got), d["scalars"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", VOXEL)
def test_voxel_gpu_matches_reference(name):
    from particuology_hydraulic_penalty_b200 import voxel_lbm

    d = golden_io.load(name)
    m = d["meta"]
    solid, dx = voxel_lbm.voxelize(d["points"], d["center"], d["size"], m["radius"], m["n"])
    assert np.array_equal(solid, d["solid"]) and np.array_equal(dx, d["dx"])
    res = voxel_lbm.run_lbm(solid, m["tau"], m["force_z"], m["steps"], return_fields=True)
    for k in ("ux", "uy", "uz"):
        assert np.array_equal(res[k], d[k]), k
    assert abs(res["permeability_lu"] - d["scalars"][3]) <= 1e-12 * abs(d["scalars"][3])
    assert res["porosity_voxel"] == d["scalars"][4]
