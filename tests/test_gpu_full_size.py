"""The headline workload at its full size, through size-independent checks.

Kerr a = 0.95, camera r = 25M, inclination 80 deg, FOV 50 deg, 1920x1080
with 2x2 regular SSAA (8,294,400 rays), RKF45 at tolerance 1e-6, three
textured spheres, the 2048x1024 starfield, FXAA.  The FP32 product render
(persistent renderer, Kahan-compensated updates) against the FP64 GPU render
of the same frame - the FP64 path is pinned to the FP64 CPU oracle ray for
ray on smaller frames (test_gpu_physical.py) - must be within 1/255 on
>= 99.9% of the pixels, the bar the workload is quoted at.  Both renders
count every ray exactly once and end none in a NaN.
"""
import numpy as np
import pytest

from conftest import pixel_rule
from parrelray_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def test_headline_frame_fp32_within_one_level_of_fp64(gpu, std_textures):
    gpu.upload_textures(std_textures)
    f32 = scenes.kerr_1080p_ssaa4()
    f64 = scenes.kerr_1080p_ssaa4(precision=abi.PREC_FP64)
    img32, _, st32 = gpu.render(f32)
    img64, _, st64 = gpu.render(f64)
    assert img32[0].shape == (1080, 1920, 3)
    for st in (st32, st64):
        assert st.rays == 1920 * 1080 * 4
        assert st.n_escaped + st.n_captured + st.n_intersection + st.n_infinite + st.n_math_error == st.rays
        assert st.n_math_error == 0
        assert st.n_intersection > 0 and st.n_captured > 0
    ok = pixel_rule(img32[0], img64[0])
    assert ok >= 0.999, ok
    # the two precisions take the same accepted steps to within a small fraction
    assert abs(st32.accepted - st64.accepted) <= 1e-3 * st64.accepted
