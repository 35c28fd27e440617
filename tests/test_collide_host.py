"""CPU check of the per-node collision header (csrc/collide.cuh) against the oracle.

The header is compiled for the host with g++ and -ffp-contract=off; its exact
FP64 variant must match the oracle's NumPy arithmetic bit for bit, its
deviation variant to round-off.
"""

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import psc_oracle as orc

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "particuology_hydraulic_penalty_b200" / "csrc"


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("shim") / "collide_shim.so"
    subprocess.run([gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I", str(CSRC),
                    str(ROOT / "tests" / "native" / "collide_host_shim.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    P = ctypes.POINTER(ctypes.c_double)
    lib.exact_collide_cells.argtypes = [P, P, P, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, P, P, P]
    lib.fast_collide_cells.argtypes = [P, P, P, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int, P, P]
    lib.fast2_collide_cells.argtypes = [P, P, P, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_int, P, P]
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def random_state(rng, ncell, amp):
    rho = 1.0 + rng.normal(0, amp, ncell)
    u = rng.normal(0, amp, (3, ncell))
    shp = (ncell, 1, 1)
    f = orc.equilibrium(rho.reshape(shp), *(u[k].reshape(shp) for k in range(3)))
    f = f + rng.normal(0, amp * 0.1, f.shape) * orc.W[:, None, None, None]
    solid = rng.choice([0.0, 1.0, 0.125, 0.5, 0.984375, rng.uniform()], size=ncell)
    us = rng.normal(0, amp, (3, ncell))
    return f, solid, us


@pytest.mark.parametrize("moving", [False, True])
@pytest.mark.parametrize("force", [(0.0, 0.0, 2e-7), (1e-6, 0.0, 0.0), (3e-7, -2e-7, 5e-7)])
def test_exact_collision_bitwise(shim, moving, force):
    rng = np.random.default_rng(5)
    ncell = 4096
    f, solid, us = random_state(rng, ncell, 1e-3)
    tau = 0.72
    shp = (ncell, 1, 1)
    post, imb = orc.collide(f, solid.reshape(shp), us.reshape(3, *shp) if moving else None, tau, force)
    rho, ux, uy, uz = orc.moments(f, force)
    fin = np.ascontiguousarray(f.reshape(19, ncell))
    fo = np.zeros_like(fin)
    io = np.zeros((3, ncell))
    mo = np.zeros((4, ncell))
    shim.exact_collide_cells(_p(fin), _p(solid), _p(np.ascontiguousarray(us)), int(moving), tau, *force, ncell,
                             _p(fo), _p(io), _p(mo))
    assert np.array_equal(fo, post.reshape(19, ncell))
    assert np.array_equal(io, imb.reshape(3, ncell))
    assert np.array_equal(mo, np.stack([rho, ux, uy, uz]).reshape(4, ncell))


@pytest.mark.parametrize("moving", [False, True])
def test_fast_collision_matches_to_roundoff(shim, moving):
    rng = np.random.default_rng(9)
    ncell = 4096
    f, solid, us = random_state(rng, ncell, 1e-3)
    tau, force = 0.8, (1e-6, 2e-7, -3e-7)
    shp = (ncell, 1, 1)
    post, imb = orc.collide(f, solid.reshape(shp), us.reshape(3, *shp) if moving else None, tau, force)
    g = np.ascontiguousarray((f - orc.W[:, None, None, None]).reshape(19, ncell))
    go = np.zeros_like(g)
    io = np.zeros((3, ncell))
    shim.fast_collide_cells(_p(g), _p(solid), _p(np.ascontiguousarray(us)), int(moving), tau, *force, ncell,
                            _p(go), _p(io))
    dev_ref = post.reshape(19, ncell) - orc.W[:, None]
    assert np.abs(go - dev_ref).max() <= 1e-15
    assert np.abs(io - imb.reshape(3, ncell)).max() <= 1e-15


@pytest.mark.parametrize("moving", [False, True])
def test_throughput_collision_matches_to_roundoff(shim, moving):
    """collide_fast2, the regrouped per-pair form the throughput kernels run (BGK), in FP64 on the
    host: post-collision deviations and IMB momentum equal the oracle's collision to round-off."""
    rng = np.random.default_rng(13)
    ncell = 4096
    f, solid, us = random_state(rng, ncell, 1e-3)
    tau, force = 0.8, (1e-6, 2e-7, -3e-7)
    shp = (ncell, 1, 1)
    post, imb = orc.collide(f, solid.reshape(shp), us.reshape(3, *shp) if moving else None, tau, force)
    g = np.ascontiguousarray((f - orc.W[:, None, None, None]).reshape(19, ncell))
    go = np.zeros_like(g)
    io = np.zeros((3, ncell))
    shim.fast2_collide_cells(_p(g), _p(solid), _p(np.ascontiguousarray(us)), int(moving), tau, 0.0, *force, ncell,
                             _p(go), _p(io))
    dev_ref = post.reshape(19, ncell) - orc.W[:, None]
    assert np.abs(go - dev_ref).max() <= 1e-15
    assert np.abs(io - imb.reshape(3, ncell)).max() <= 1e-15


def test_throughput_trt_collision_matches_oracle_extension(shim):
    """The same form with tau_minus > 0 equals the oracle's TRT extension (static solid) to round-off."""
    from particuology_hydraulic_penalty_b200.engine import trt_tau_minus

    rng = np.random.default_rng(17)
    ncell = 4096
    f, solid, us = random_state(rng, ncell, 1e-3)
    tau, force = 0.8, (1e-6, 2e-7, -3e-7)
    tm = trt_tau_minus(tau)
    shp = (ncell, 1, 1)
    g4 = f - orc.W[:, None, None, None]
    ref = orc.collide_trt_deviation(g4, solid.reshape(shp), tau, tm, force).reshape(19, ncell)
    g = np.ascontiguousarray(g4.reshape(19, ncell))
    go = np.zeros_like(g)
    io = np.zeros((3, ncell))
    shim.fast2_collide_cells(_p(g), _p(solid), _p(np.ascontiguousarray(us)), 0, tau, tm, *force, ncell, _p(go), _p(io))
    assert np.abs(go - ref).max() <= 1e-15
