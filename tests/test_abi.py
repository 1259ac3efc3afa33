"""The C-ABI library loads, exports every symbol include/prr.h declares, and
its structs have the layout the Python binding assumes.  No GPU needed."""
import ctypes as C

import pytest

from parrelray_b200 import abi


def test_library_exports_every_declared_function(built):
    lib = abi.load()
    names = abi.header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared in include/prr.h but not exported: {missing}"
    assert set(names) <= set(abi.SIGNATURES), "binding lacks a signature for a declared function"


def test_struct_layouts_match(built):
    lib = abi.load()
    assert lib.prr_sizeof(0) == C.sizeof(abi.FrameDesc)
    assert lib.prr_sizeof(1) == C.sizeof(abi.Stats)
    assert lib.prr_sizeof(2) == C.sizeof(abi.LaunchConfig)
    assert lib.prr_sizeof(3) == C.sizeof(abi.Sphere)
    assert lib.prr_sizeof(4) == C.sizeof(abi.EmissionDesc)
    assert lib.prr_sizeof(5) == C.sizeof(abi.PlasmaDesc)
    assert lib.prr_sizeof(99) == 0


def test_version_and_status_strings(built):
    lib = abi.load()
    assert lib.prr_abi_version() == 4
    assert lib.prr_status_string(abi.OK) == b"ok"
    assert b"device" in lib.prr_status_string(abi.ERR_NO_DEVICE)


def test_defaults_follow_the_reference_deck(built):
    d = abi.defaults()
    # input/sim.params:10-13 and metrics/schwarzschild.cuh:70
    assert (d.h, d.hmin, d.hmax) == pytest.approx((0.01, 1e-4, 0.1))
    assert d.eps == pytest.approx(1e-3)
    assert d.horizon_eps == pytest.approx(1e-3)
    assert d.solver == abi.SOLVER_RKF45 and d.max_steps == 10000


def test_library_free_defaults_equal_the_library_defaults(built):
    """scenes builds frames with abi.fill_defaults (no library load); it must write the same bytes
    as prr_frame_desc_defaults."""
    a = bytes(abi.defaults())
    b = bytes(abi.fill_defaults(abi.FrameDesc()))
    assert a == b


def test_null_arguments_are_rejected_without_a_device(built):
    lib = abi.load()
    assert lib.prr_create(0, None) == abi.ERR_INVALID
    assert lib.prr_render(None, None, 0, None, None, None) == abi.ERR_INVALID
    assert lib.prr_upload_texture(None, 0, None, 0, 0) == abi.ERR_INVALID
    assert lib.prr_make_texture(5, 0, 16, 16, None) == abi.ERR_INVALID


def test_no_device_reports_no_device(built):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    assert abi.load().prr_create(0, C.byref(h)) == abi.ERR_NO_DEVICE
    assert not h.value
