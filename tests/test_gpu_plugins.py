"""Metric plug-ins on the GPU: a reference-style metric header compiled
UNCHANGED against the compatibility tree (parrelray_b200/compat) and loaded
with prr_load_metric_plugin renders what the reference renders with it.

* The Kerr plug-in header shipped in compat/metrics/kerr.cuh, and - where the
  plug-in libraries were built from the reference tree - the reference's own
  metrics/schwarzschild.cuh and metrics/flat.cuh, against the golden outputs
  of the reference's frame pipeline (tests/golden/*.npz, made by the reference
  sources with the same headers): the REFERENCE-mode bars (outcome for
  >= 99.5% of rays, image within 1/255 on >= 99.9% of pixels).
* A plug-in and the built-in REFERENCE path for the same metric agree ray for
  ray.
* The reference's spherical-coordinate header metrics/"schwarzschild - sph.cuh"
  (states (r, theta, phi, t), built with SPHERICAL) against the reference's
  own frame pipeline built with the same header and switch
  (tests/golden/plugin_sph_*.npz).
* PHYSICAL mode through a header's hooks on the persistent scheduler: the
  reference's own metrics/schwarzschild.cuh renders the single-frame
  Schwarzschild workload (320x180, tolerance 1e-6) within 1/255 of the FP64
  host oracle on >= 99.9% of pixels, and the shipped Kerr header renders the
  Kerr test frame (a = 0.95, 2x2 SSAA, three spheres) to the same bar.
"""
import numpy as np
import pytest

from conftest import pixel_rule, quantize
from parrelray_b200 import abi
from parrelray_b200.abi import LIB_PATH
from test_oracle_golden import load_case

pytestmark = pytest.mark.gpu

PLUGINS = {"kerr": ("kerr_48x27_s1",), "schwarzschild": ("schw_160x90_s1", "schw_64x36_s4"),
           "flat": ("flat_64x36_s1",)}


def plugin_path(name):
    return LIB_PATH.parent / f"libprr_metric_{name}.so"


def _cases():
    out = []
    for name, cases in PLUGINS.items():
        for c in cases:
            out.append((name, c))
    return out


@pytest.mark.parametrize("plugin,case", _cases())
def test_plugin_matches_reference_golden(gpu, plugin, case):
    p = plugin_path(plugin)
    if not p.exists():
        if plugin == "kerr":
            pytest.fail("the Kerr plug-in ships with the repository and must be built")
        pytest.skip(f"{p.name} is built only where the reference's headers are available")
    mid = gpu.load_metric_plugin(p)
    assert mid >= abi.METRIC_PLUGIN0
    d, tex, z = load_case(case)
    builtin_metric = d.metric
    gpu.upload_textures(tex)
    d.metric = mid
    state, rgb, stats = gpu.trace_rays(d)
    assert stats.rays == d.nrays and stats.attempts > 0
    ref = z["state"]
    same = state[:, 2] == ref[:, 2]
    assert same.mean() >= 0.995, same.mean()
    imgs, _, _ = gpu.render(d)
    npx = d.width * d.height
    ok = pixel_rule(imgs[0], quantize(z["image"]))
    assert ok >= min(0.999, 1 - 1.0 / npx - 1e-12), ok
    # against the built-in REFERENCE path of the same metric: the same
    # arithmetic for Schwarzschild and flat (ray for ray); the built-in Kerr
    # evaluates the geodesic by a different contraction than the plug-in's
    # Christoffel table, so only outcomes are compared there
    d.metric = builtin_metric
    bstate, brgb, _ = gpu.trace_rays(d)
    assert np.mean(bstate[:, 2] == state[:, 2]) >= 0.995
    if plugin != "kerr":
        exact = np.all(bstate[:, :11] == state[:, :11], axis=1)
        assert exact.mean() >= 0.99, exact.mean()
        assert np.mean(np.abs(brgb - rgb).max(axis=1) <= 1 / 255) >= 0.995


def test_plugin_loading_rules(gpu, small_textures):
    p = plugin_path("kerr")
    a = gpu.load_metric_plugin(p)
    assert gpu.load_metric_plugin(p) == a  # same path, same id
    with pytest.raises(abi.PrrError) as e:
        gpu.load_metric_plugin(LIB_PATH)  # a library without the plug-in entry points
    assert e.value.status == abi.ERR_INVALID
    with pytest.raises(abi.PrrError) as e:
        gpu.load_metric_plugin(LIB_PATH.parent / "libprr_metric_nosuch.so")
    assert e.value.status == abi.ERR_IO
    from parrelray_b200 import scenes

    gpu.upload_textures(small_textures)
    d = scenes.schwarzschild_320(precision=abi.PREC_FP64)
    d.metric = a  # PHYSICAL mode in FP64: a header's getGeod is FP32
    with pytest.raises(abi.PrrError) as e:
        gpu.render(d)
    assert e.value.status == abi.ERR_INVALID
    b = scenes.schwarzschild_320()
    d = scenes.schwarzschild_320()
    d.metric = a
    with pytest.raises(abi.PrrError) as e:  # plug-in and built-in frames in one call
        gpu.render([d, b])
    assert e.value.status == abi.ERR_INVALID
    d.metric = abi.METRIC_PLUGIN0 + 7  # not loaded
    d.mode = abi.MODE_REFERENCE
    with pytest.raises(abi.PrrError) as e:
        gpu.render(d)
    assert e.value.status == abi.ERR_INVALID


def test_reference_alternative_cartesian_header(gpu, small_textures):
    """The reference's alternative header metrics/"schwarzschild - cart.cuh" (Christoffel tables, not
    selected by its main/metric.h), compiled unchanged as a plug-in, against the reference's own host
    build with that header selected, live on the same deck (its rays end in MATH_ERROR at the first
    step in the reference too: the plug-in reproduces the header as written)."""
    from pathlib import Path

    from oracles import RefHost, ref_available, write_deck
    from parrelray_b200 import scenes

    p = plugin_path("schwarzschildcart")
    if not p.exists() or not ref_available("cart"):
        pytest.skip("built only where the reference's headers are available")
    sph = [(*scenes.orbit_point(10.0, 60.0), 1.5, scenes.SPHERE_ID0), (*scenes.orbit_point(12.0, 200.0), 2.0, 2)]
    d = scenes.make_frame(64, 36, r=30.0, incl_deg=85.0, fov_deg=60.0, metric=abi.METRIC_SCHWARZSCHILD, mass=1.0,
                          spheres=sph, mode=abi.MODE_REFERENCE, eps=1e-3, horizon_eps=0.001)
    _, a_deg, b_deg = scenes.camera_pose(30.0, 85.0)
    deck = write_deck(Path("/tmp/prrcartgpu"), d, small_textures, fov_deg=60.0, a_deg=a_deg, b_deg=b_deg)
    ref = RefHost("cart")
    assert ref.load(deck) == 1
    z = ref.frame(0)
    gpu.upload_textures(small_textures)
    d.metric = gpu.load_metric_plugin(p)
    state, rgb, _ = gpu.trace_rays(d)
    assert np.mean(state[:, 2] == z["state"][:, 2]) >= 0.995
    imgs, _, _ = gpu.render(d)
    assert pixel_rule(imgs[0], quantize(z["image"])) >= 0.999


@pytest.mark.parametrize("case", ["plugin_sph_64x36_s1", "plugin_sph_32x18_s4"])
def test_reference_spherical_header(gpu, case):
    """metrics/"schwarzschild - sph.cuh" compiled unchanged with SPHERICAL: rays start at the camera's
    spherical position with the spherical rates of the pin-hole direction (kernels/solver.cuh:34-37),
    the header's pole flip and angle wrapping run in User_ENDLOOP, and its rayToRGB looks the sky up
    at the final (theta, phi) (main/base.h:68-117).  Bars: the REFERENCE-mode ones; escape angles
    within 1e-3 rad for >= 99% of the rays that escape in both."""
    p = plugin_path("schwarzschildsph")
    if not p.exists():
        pytest.skip(f"{p.name} is built only where the reference's headers are available")
    d, tex, z = load_case(case)
    gpu.upload_textures(tex)
    d.metric = gpu.load_metric_plugin(p)
    state, rgb, stats = gpu.trace_rays(d)
    ref = z["state"]
    assert stats.rays == d.nrays and stats.attempts > 0
    assert np.mean(state[:, 2] == ref[:, 2]) >= 0.995
    esc = (ref[:, 2] == abi.RESULT_SUCCESS) & (ref[:, 3] >= 100.0) & (state[:, 3] >= 100.0)
    assert esc.sum() > 0.3 * d.nrays
    dth = np.abs(state[esc, 4] - ref[esc, 4])
    dph = np.abs(np.angle(np.exp(1j * (state[esc, 5].astype(np.float64) - ref[esc, 5]))))
    assert np.mean((dth <= 1e-3) & (dph <= 1e-3)) >= 0.99, (dth.max(), dph.max())
    cap = (ref[:, 2] == abi.RESULT_SUCCESS) & (ref[:, 3] < 3.0)
    assert np.mean(state[cap, 3] < 3.0) >= 0.99
    assert np.mean(np.abs(rgb - z["rgb"]).max(axis=1) <= 1 / 255) >= 0.99
    imgs, _, _ = gpu.render(d)
    npx = d.width * d.height
    assert pixel_rule(imgs[0], quantize(z["image"])) >= min(0.999, 1 - 1.0 / npx - 1e-12)


def test_reference_schwarzschild_header_physical_mode(gpu, oracle, std_textures):
    """The reference's own metrics/schwarzschild.cuh, compiled unchanged, renders the single-frame
    Schwarzschild workload (M = 1, camera r = 30M, inclination 85 deg, FOV 60 deg, 320x180, one
    sphere R = 1M at r = 10M, tolerance 1e-6) in PHYSICAL mode on the persistent scheduler; the
    header's User_ENDLOOP stops at r <= rs + 0.001 (metrics/schwarzschild.cuh:70), so the oracle
    stops there too."""
    from parrelray_b200 import scenes

    p = plugin_path("schwarzschild")
    if not p.exists():
        pytest.skip(f"{p.name} is built only where the reference's headers are available")
    d = scenes.schwarzschild_320(horizon_eps=0.001)
    gpu.upload_textures(std_textures)
    d.metric = gpu.load_metric_plugin(p)
    imgs, _, stats = gpu.render(d)
    assert stats.rays == 57600 and stats.attempts >= stats.accepted > 0
    assert stats.n_infinite == 0 and stats.n_math_error == 0
    assert stats.n_intersection > 0 and stats.n_captured > 0 and stats.n_escaped > 0
    d64 = scenes.schwarzschild_320(horizon_eps=0.001, precision=abi.PREC_FP64)
    _, _, ref = oracle.render(d64, std_textures, precision=1)
    ok = pixel_rule(imgs[0], quantize(ref))
    assert ok >= 0.999, ok
    # the built-in PHYSICAL renderer of the same metric agrees too
    b = scenes.schwarzschild_320(horizon_eps=0.001)
    bimg, _, _ = gpu.render(b)
    assert pixel_rule(imgs[0], bimg[0]) >= 0.999


def test_shipped_kerr_header_physical_mode(gpu, oracle, small_textures):
    """The Kerr header shipped in compat/metrics/kerr.cuh (Christoffel-table geodesic, as a plug-in
    author would write it) in PHYSICAL mode: a = 0.95, 64x36 with 2x2 SSAA and FXAA, three spheres,
    tolerance 1e-6, against the FP64 host oracle.  Its User_ENDLOOP stops at r <= r_+ + 0.001."""
    from parrelray_b200 import scenes

    sph = [(*scenes.orbit_point(orb, ph), rad, scenes.SPHERE_ID0 + k)
           for k, (rad, orb, ph) in enumerate(scenes.KERR_1080P_SPHERES)]
    kw = dict(r=25.0, incl_deg=80.0, fov_deg=50.0, metric=abi.METRIC_KERR, mass=1.0, spin=0.95, samples=4,
              fxaa=True, spheres=sph, horizon_eps=0.001)
    d = scenes.make_frame(64, 36, **kw)
    gpu.upload_textures(small_textures)
    d.metric = gpu.load_metric_plugin(plugin_path("kerr"))
    state, rgb, stats = gpu.trace_rays(d)
    assert stats.rays == d.nrays and stats.attempts > 0
    d64 = scenes.make_frame(64, 36, precision=abi.PREC_FP64, **kw)
    st64, _, ref = oracle.render(d64, small_textures, precision=1)
    assert np.mean(state[:, 2] == st64[:, 2]) >= 0.995
    imgs, _, _ = gpu.render(d)
    ok = pixel_rule(imgs[0], quantize(ref))
    assert ok >= 0.999 - 1.0 / (d.width * d.height), ok
