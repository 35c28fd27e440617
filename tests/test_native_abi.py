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
    assert "psc_step_windows" in names and "psc_geometry_build" in names
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
    assert lib.psc_step_windows(0, None, 1, 1, 1, 0, None) == nat.PSC_E_INVALID
    assert lib.psc_step_windows(9, None, 1, 1, 1, 0, None) == nat.PSC_E_INVALID
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


def _config(**kw):
    c = nat.PscConfig()
    c.nx = c.ny = c.nz = 16
    c.subsamples = 4
    c.store = nat.STORE_F32
    c.tau = 0.8
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def test_handle_layer_layout(lib):
    assert lib.psc_config_size() == ctypes.sizeof(nat.PscConfig)
    assert lib.psc_diag_size() == ctypes.sizeof(nat.PscDiag)
    assert lib.psc_status_size() == ctypes.sizeof(nat.PscStatus)


@pytest.mark.parametrize("kw, code, words", [
    ({"nx": 0}, nat.PSC_E_INVALID, b"extents"),
    ({"store": 9}, nat.PSC_E_INVALID, b"store"),
    ({"subsamples": 7}, nat.PSC_E_UNSUPPORTED, b"uint8"),
    ({"tau": -1.0}, nat.PSC_E_INVALID, b"tau"),
    ({"store": nat.STORE_F64_EXACT, "tau_minus": 1.0}, nat.PSC_E_UNSUPPORTED, b"TRT"),
    ({"nx": 1000, "ny": 1000, "nz": 200}, nat.PSC_E_UNSUPPORTED, b"2^31"),
])
def test_handle_config_rejected_before_device_use(lib, kw, code, words):
    h = ctypes.c_void_p()
    cfg = _config(**kw)
    assert lib.psc_create(ctypes.byref(cfg), ctypes.byref(h)) == code
    assert words in lib.psc_last_error()
    assert not h.value


def test_handle_null_arguments(lib):
    h = ctypes.c_void_p()
    assert lib.psc_create(None, ctypes.byref(h)) == nat.PSC_E_INVALID
    st = nat.PscStatus()
    assert lib.psc_step(None, 1, 0, ctypes.byref(st)) == nat.PSC_E_INVALID
    assert lib.psc_get_fields(None, 0, None) == nat.PSC_E_INVALID
    assert lib.psc_set_particles(None, None, 0) == nat.PSC_E_INVALID
    assert lib.psc_destroy(None) == nat.PSC_OK
    assert lib.psc_batch_destroy(None) == nat.PSC_OK


def test_batch_config_mismatch_rejected(lib):
    cfgs = (nat.PscConfig * 2)(_config(), _config(store=nat.STORE_F64))
    b = ctypes.c_void_p()
    assert lib.psc_batch_create(cfgs, 2, None, 20, ctypes.byref(b)) == nat.PSC_E_INVALID
    assert b"same store" in lib.psc_last_error()
    cfgs = (nat.PscConfig * 2)(_config(), _config())
    assert lib.psc_batch_create(cfgs, 2, None, 3, ctypes.byref(b)) == nat.PSC_E_INVALID
    assert b"even" in lib.psc_last_error()


def test_row_planner_rejects_open_windows(lib):
    w = (nat.PscWindow * 1)()
    w[0].nx, w[0].ny, w[0].nz = 16, 16, 16
    w[0].flags = nat.WIN_OPEN_X
    total, sb = ctypes.c_int64(0), ctypes.c_int32(0)
    assert lib.psc_plan_row_tiles(w, 1, 0, 4, ctypes.byref(total), ctypes.byref(sb)) == nat.PSC_E_UNSUPPORTED
    assert b"periodic" in lib.psc_last_error()


def test_open_window_config_checked(lib):
    h = ctypes.c_void_p()
    cfg = _config(open_x=1, inlet_rho=0.0)
    assert lib.psc_create(ctypes.byref(cfg), ctypes.byref(h)) == nat.PSC_E_INVALID
    assert b"inlet" in lib.psc_last_error()


def test_pair_planner_needs_even_nz(lib):
    w = (nat.PscWindow * 2)()
    w[0].nx, w[0].ny, w[0].nz = 8, 8, 8
    w[1].nx, w[1].ny, w[1].nz = 8, 8, 9
    total = ctypes.c_int64(0)
    assert lib.psc_plan_pair_tiles(w, 2, ctypes.byref(total)) == nat.PSC_E_UNSUPPORTED
    assert b"even nz" in lib.psc_last_error()
    w[1].nz = 10
    assert lib.psc_plan_pair_tiles(w, 2, ctypes.byref(total)) == nat.PSC_OK
    assert w[0].tile_cells == 512 and total.value == 1 + (640 + 511) // 512
