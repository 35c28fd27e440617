"""GPU check of the correctly rounded division by a known divisor (xdiv_r, csrc/d3q19.cuh) that the
exact FP64 kernels use in place of x / c_s^2, x / c_s^4, x / tau and x / rho: bit for bit against
CUDA's IEEE division __ddiv_rn, on 2^33 random x per constant divisor (random sign and significand,
exponents over the whole fast-path range and near 1), on random relaxation times and densities, and
on signed zeros, subnormals, the range edges, infinities and NaN.  The helper is built here with nvcc
(tests/native/div_check.cu)."""

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "particuology_hydraulic_penalty_b200" / "csrc"
CS2 = 1.0 / 3.0


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    out = tmp_path_factory.mktemp("divgpu") / "div_check_gpu.so"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared", "-I", str(CSRC),
                    str(ROOT / "tests" / "native" / "div_check.cu"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.div_check_gpu.restype = ctypes.c_longlong
    lib.div_check_gpu.argtypes = [ctypes.c_double, ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_int,
                                  ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.div_list_gpu.restype = ctypes.c_int
    P = ctypes.POINTER(ctypes.c_double)
    lib.div_list_gpu.argtypes = [ctypes.c_double, P, ctypes.c_int, P, P]
    return lib


def _random(lib, y, n, seed, emin, emax):
    first = ctypes.c_double(0.0)
    bad = lib.div_check_gpu(y, n, seed, emin, emax, ctypes.byref(first))
    assert bad >= 0, "CUDA error in the check kernel"
    return bad, first.value


@pytest.mark.parametrize("y", [CS2, CS2 * CS2])
def test_constant_divisors(lib, y):
    for seed, (emin, emax) in enumerate([(-900, 900), (-40, 3), (-3, 0)]):
        bad, x = _random(lib, y, 1 << 33, 17 + seed, emin, emax)
        assert bad == 0, (y, emin, emax, x)


def test_relaxation_times_and_densities(lib):
    rng = np.random.default_rng(11)
    taus = [0.5000001, 0.51, 0.6, 0.72, 0.8, 1.0, 1.7, 2.5, 7.3, 255.9]
    rhos = list(rng.uniform(0.9, 1.1, 8)) + [1.0 - 2.0 ** -52, 1.0 + 2.0 ** -52]
    for k, y in enumerate(taus + rhos):
        bad, x = _random(lib, float(y), 1 << 30, 101 + k, -60, 3)
        assert bad == 0, (y, x)


@pytest.mark.parametrize("y", [CS2, CS2 * CS2, 0.72, 1.0, 300.0, 2.0 ** -9, -0.8, 2.0 ** 8, 2.0 ** -8])
def test_special_values(lib, y):
    tiny = np.finfo(float).tiny
    xs = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, -5e-324, tiny, -tiny, tiny * 3.5, 2.0 ** -900,
                   -2.0 ** -900, np.nextafter(2.0 ** -900, 0.0), 2.0 ** 900, np.nextafter(2.0 ** 900, np.inf),
                   1.7976931348623157e308, -1.7976931348623157e308, 1.0, -1.0, 1e-300, 1e300, 3.0, 1.0 / 3.0],
                  dtype=float)
    out, ref = np.empty_like(xs), np.empty_like(xs)
    P = ctypes.POINTER(ctypes.c_double)
    assert lib.div_list_gpu(y, xs.ctypes.data_as(P), len(xs), out.ctypes.data_as(P), ref.ctypes.data_as(P)) == 0
    same = (out.view(np.uint64) == ref.view(np.uint64)) | (np.isnan(out) & np.isnan(ref))
    assert same.all(), xs[~same]
