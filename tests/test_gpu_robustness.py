"""Error paths of the C ABI on a device: every bad descriptor is rejected
with PRR_ERR_INVALID and a message; the device watchdog ends a render early
with PRR_ERR_TIMEOUT and leaves the context usable; failures are made on the
host or by a short cycle budget, never by faulting the GPU."""
import ctypes as C

import numpy as np
import pytest

from parrelray_b200 import PrrError, abi, scenes

pytestmark = pytest.mark.gpu


def good():
    return scenes.make_frame(16, 9, r=25.0, incl_deg=80.0, fov_deg=50.0, metric=abi.METRIC_KERR, spin=0.5)


@pytest.mark.parametrize("field,value", [
    ("width", 0), ("height", -1), ("samples", 0), ("samples", 2), ("metric", 7), ("mass", -1.0),
    ("spin", 2.0), ("solver", 1), ("mode", 5), ("precision", 9), ("hmin", 0.0), ("hmax", 1e-5),
    ("rout", 0.0), ("max_steps", 0), ("background_id", 31), ("nspheres", 9), ("vfov", 0.0),
])
def test_invalid_descriptor_is_rejected(gpu, small_textures, field, value):
    gpu.upload_textures(small_textures)
    d = good()
    setattr(d, field, value)
    if field == "samples" and value == 2:
        d.ssaa = abi.SSAA_REGULAR  # not a perfect square
    with pytest.raises(PrrError) as e:
        gpu.render(d)
    assert e.value.status == abi.ERR_INVALID
    assert str(e.value)


def test_reference_mode_rejects_fp64(gpu):
    d = good()
    d.mode = abi.MODE_REFERENCE
    d.precision = abi.PREC_FP64
    with pytest.raises(PrrError):
        gpu.render(d)


def test_bad_texture_upload(gpu):
    with pytest.raises(PrrError):
        gpu.upload_texture(40, np.zeros((4, 4, 4), np.uint8))


def test_watchdog_times_out_and_context_survives(gpu, small_textures):
    gpu.upload_textures(small_textures)
    d = scenes.make_frame(256, 144, r=25.0, incl_deg=80.0, fov_deg=50.0, metric=abi.METRIC_KERR, spin=0.9)
    gpu.set_option(abi.OPT_WATCHDOG_CYCLES, 20000)
    try:
        with pytest.raises(PrrError) as e:
            gpu.render(d)
        assert e.value.status == abi.ERR_TIMEOUT
    finally:
        gpu.set_option(abi.OPT_WATCHDOG_CYCLES, 0)
    imgs, _, stats = gpu.render(good())
    assert stats.rays == 16 * 9 and imgs[0].shape == (9, 16, 3)
