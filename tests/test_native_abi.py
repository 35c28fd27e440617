"""CPU checks of the C ABI: the library loads, exports every declared symbol,
and its struct layout matches the ctypes mirror.  No device calls."""

import ctypes
import re

import pytest

from particuology_hydraulic_penalty_b200 import _native as nat
from particuology_hydraulic_penalty_b200 import build as pbuild


@pytest.fixture(scope="module")
def lib():
    pbuild.build()
    return nat.load()


def declared_functions():
    text = nat.HEADER_PATH.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(psc_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "psc_step" in names and "psc_geometry_build" in names
    assert len(names) >= 14


def test_every_declared_symbol_is_exported(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_ctypes_signatures_cover_header():
    assert set(declared_functions()) <= set(nat.SIGNATURES)


def test_struct_layout_matches(lib):
    assert lib.psc_window_size() == ctypes.sizeof(nat.PscWindow)
    assert lib.psc_geometry_size() == ctypes.sizeof(nat.PscGeometry)
    assert lib.psc_abi_version() == nat.ABI_VERSION


def test_host_only_entry_points(lib):
    # psc_plan_tiles is pure host logic
    w = (nat.PscWindow * 2)()
    w[0].nx, w[0].ny, w[0].nz = 20, 20, 20
    w[1].nx, w[1].ny, w[1].nz = 7, 5, 3
    total = ctypes.c_int64(0)
    assert lib.psc_plan_tiles(w, 2, 0, ctypes.byref(total)) == nat.PSC_OK
    assert w[0].tile_begin == 0 and w[0].tile_count == (8000 + 255) // 256
    assert w[1].tile_begin == w[0].tile_count and w[1].tile_count == 1
    assert total.value == w[0].tile_count + 1
    # invalid extents are rejected with a message, no exception
    w[1].nz = 0
    assert lib.psc_plan_tiles(w, 2, 0, ctypes.byref(total)) == nat.PSC_E_INVALID
    assert b"extents" in lib.psc_last_error()
    assert lib.psc_plan_tiles(w, 2, 100, ctypes.byref(total)) == nat.PSC_E_UNSUPPORTED
    assert lib.psc_scan_tmp_bytes(10 ** 6) > 0


def test_null_arguments_rejected_without_device(lib):
    assert lib.psc_step(0, None, 1, 1, 1, 0, None) == nat.PSC_E_INVALID
    assert lib.psc_step(9, None, 1, 1, 1, 0, None) == nat.PSC_E_INVALID
    assert lib.psc_init_equilibrium(0, 1.0, None, 10, None) == nat.PSC_E_INVALID
    assert lib.psc_geometry_plan(None, None) == nat.PSC_E_INVALID
    assert lib.psc_stream_push(0, 1.0, None, None, 4, 4, 4, None) == nat.PSC_E_INVALID


def test_product_requires_cuda():
    import torch

    from particuology_hydraulic_penalty_b200 import PscD3Q19, Particle3D

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(RuntimeError, match="CUDA"):
        PscD3Q19(8, [Particle3D(4.0, 4.0, 4.0, 2.0)])
