"""CPU check of the correctly rounded division by a known divisor (xdiv_r in csrc/d3q19.cuh) that the
exact FP64 kernels use for x / c_s^2, x / c_s^4, x / tau and x / rho.

The header is compiled for the host with g++ and compared bit for bit with the host's IEEE binary64
division (x / y, correctly rounded) on random x over the whole exponent range the fast path covers,
on the edges of that range, and on signed zeros, subnormals, infinities and NaN, for the divisors the
kernels use: c_s^2 and c_s^4 (constants), relaxation times tau, and densities rho near 1.  Any out-of-
range divisor takes the IEEE division."""

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "particuology_hydraulic_penalty_b200" / "csrc"
CS2 = 1.0 / 3.0
DIVISORS = [CS2, CS2 * CS2, 0.5000001, 0.51, 0.6, 0.72, 0.8, 1.0, 1.2345678901234567, 1.7, 3.0, 255.9, 2.0 ** -8,
            2.0 ** 8, 0.9999999999999999, 1.0000000000000002, 0.97, 1.03]


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("div") / "div_check.so"
    subprocess.run([gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I", str(CSRC),
                    str(ROOT / "tests" / "native" / "div_check.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.div_check_random.restype = ctypes.c_longlong
    lib.div_check_random.argtypes = [ctypes.c_double, ctypes.c_longlong, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double)]
    lib.div_check_list.restype = ctypes.c_longlong
    lib.div_check_list.argtypes = [ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.c_longlong,
                                   ctypes.POINTER(ctypes.c_double)]
    return lib


@pytest.mark.parametrize("y", DIVISORS)
def test_random_x_bitwise(lib, y):
    bad = ctypes.c_double(0.0)
    for seed, (emin, emax) in enumerate([(-900, 900), (-30, 5), (-2, 1)]):
        n = lib.div_check_random(y, 400000, 1000 + seed, emin, emax, ctypes.byref(bad))
        assert n == 0, (y, emin, emax, bad.value)


def test_random_density_divisors(lib):
    rng = np.random.default_rng(3)
    bad = ctypes.c_double(0.0)
    for y in rng.uniform(0.95, 1.05, 40):
        assert lib.div_check_random(float(y), 50000, int(rng.integers(1 << 62)), -60, 2, ctypes.byref(bad)) == 0


@pytest.mark.parametrize("y", [CS2, CS2 * CS2, 0.72, 1.0, 300.0, 2.0 ** -9, -0.8])
def test_special_values(lib, y):
    tiny = np.finfo(float).tiny
    xs = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, -5e-324, tiny, -tiny, tiny * 3.5, 2.0 ** -900,
                   -2.0 ** -900, np.nextafter(2.0 ** -900, 0.0), 2.0 ** 900, np.nextafter(2.0 ** 900, np.inf),
                   1.7976931348623157e308, -1.7976931348623157e308, 1.0, -1.0, 1e-300, 1e300, 3.0, 1.0 / 3.0],
                  dtype=float)
    out = np.empty_like(xs)
    n = lib.div_check_list(y, xs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(xs),
                           out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert n == 0
    assert np.signbit(out[1]) != np.signbit(out[0])  # the sign of zero survives
