"""Pins the CPU restatement (oracle/prr_oracle.cpp) to the reference.

1. Against the committed golden fixtures, which were produced by the
   reference's own sources (tests/golden/make_golden.py): bit-exact per-ray
   states, colours, SSAA combine and FXAA.
2. Where the reference tree is mounted, against a live run of the reference
   host build on further seeded decks (Euler and RKF45).
"""
import json
from pathlib import Path

import numpy as np
import pytest

from parrelray_b200 import abi, scenes

GOLDEN = Path(__file__).parent / "golden"
# the built-in metrics; plugin_* fixtures hold a reference metric header's own
# outputs (tests/test_gpu_plugins.py) and have no restatement here; full_*
# fixtures are the full-size single-frame workload in slim form
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz") if not p.stem.startswith(("plugin_", "full_")))
FULL_CASES = sorted(p.stem for p in GOLDEN.glob("full_*.npz"))


def load_case(name):
    from golden.make_golden import ALL_CASES as SPECS, case_frame, case_textures

    z = np.load(GOLDEN / f"{name}.npz")
    d, meta = case_frame(SPECS[name])
    assert json.loads(str(z["meta"]))["W"] == meta["W"]
    return d, case_textures(SPECS[name]), z


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_bitwise(oracle, name):
    d, tex, z = load_case(name)
    st, rgb = oracle.trace(d, tex)
    ref_state = z["state"]
    mine = st[:, :11].astype(np.float32)
    assert np.array_equal(mine, ref_state, equal_nan=True)
    assert np.array_equal(rgb, z["rgb"], equal_nan=True)
    img = oracle.post(rgb, d.width, d.height, d.samples, False)
    assert np.array_equal(img, z["image"])
    fx = oracle.post(rgb, d.width, d.height, d.samples, True)
    assert np.array_equal(fx[1:-1, 1:-1], z["fxaa"][1:-1, 1:-1])


@pytest.mark.parametrize("name", FULL_CASES)
def test_oracle_reproduces_full_size_reference_frame(oracle, name):
    """The 320x180 single-frame workload in the reference's own solver: the restatement gives
    the same result, quantised direction and 8-bit colour for every one of its 57,600 rays."""
    from golden.make_golden import slim

    d, tex, z = load_case(name)
    st, rgb = oracle.trace(d, tex)
    mine = slim(st[:, :11].astype(np.float32), rgb)
    for k in ("result", "direction", "rgb8"):
        assert np.array_equal(mine[k], z[k]), k
    res = np.bincount(z["result"].astype(int), minlength=5)
    assert res[abi.RESULT_SUCCESS] > 0 and res[abi.RESULT_INTERSECTION] > 0


def test_euler_case_exercises_the_euler_solver():
    from golden.make_golden import ALL_CASES, case_frame

    d, meta = case_frame(ALL_CASES["euler_64x36_s1"])
    assert d.solver == abi.SOLVER_EULER and meta["solver"] == "euler"
    z = np.load(GOLDEN / "euler_64x36_s1.npz")
    res = np.bincount(z["state"][:, 2].astype(int), minlength=5)
    assert res[abi.RESULT_SUCCESS] > 0 and res[abi.RESULT_INTERSECTION] > 0


@pytest.mark.parametrize("name", CASES)
def test_golden_cases_exercise_the_hooks(name):
    z = np.load(GOLDEN / f"{name}.npz")
    res = np.bincount(z["state"][:, 2].astype(int), minlength=5)
    assert res[abi.RESULT_SUCCESS] > 0
    assert res[abi.RESULT_INTERSECTION] > 0, "every golden case has visible spheres"


def _live_case(tmp_base, metric_tag, metric, W, H, S, eps, solver, seed):
    from oracles import RefHost, write_deck

    rng = np.random.default_rng(seed)
    r = float(rng.uniform(15, 40))
    inc = float(rng.uniform(20, 89))
    fov = float(rng.uniform(30, 70))
    spheres = [(*scenes.orbit_point(float(rng.uniform(6, 14)), float(rng.uniform(0, 360))),
                float(rng.uniform(0.5, 2.0)), 1 + k) for k in range(int(rng.integers(1, 4)))]
    spin = float(rng.uniform(0, 0.99)) if metric == abi.METRIC_KERR else 0.0
    d = scenes.make_frame(W, H, r=r, incl_deg=inc, fov_deg=fov, metric=metric, mass=1.0, spin=spin, samples=S,
                          mode=abi.MODE_REFERENCE, eps=eps, horizon_eps=0.001, spheres=spheres)
    d.solver = abi.SOLVER_EULER if solver == "euler" else abi.SOLVER_RKF45
    _, a_deg, b_deg = scenes.camera_pose(r, inc)
    return d, a_deg, b_deg, fov


@pytest.mark.parametrize("seed,metric_tag,metric,S,solver", [
    (11, "schw", abi.METRIC_SCHWARZSCHILD, 1, "rkf"),
    (12, "schw", abi.METRIC_SCHWARZSCHILD, 4, "rkf"),
    (13, "schw", abi.METRIC_SCHWARZSCHILD, 1, "euler"),
    (14, "flat", abi.METRIC_FLAT, 1, "rkf"),
    (15, "kerr", abi.METRIC_KERR, 1, "rkf"),
])
def test_oracle_matches_live_reference(oracle, small_textures, seed, metric_tag, metric, S, solver):
    from oracles import RefHost, ref_available, write_deck

    if not ref_available(metric_tag):
        pytest.skip("reference host build not available (reference tree absent)")
    d, a_deg, b_deg, fov = _live_case(None, metric_tag, metric, 40, 24, S, 1e-3, solver, seed)
    deck = write_deck(Path("/tmp/prrlive"), d, small_textures, fov_deg=fov, a_deg=a_deg, b_deg=b_deg, solver=solver)
    ref = RefHost(metric_tag)
    assert ref.load(deck) == 1
    out = ref.frame(0)
    st, rgb = oracle.trace(d, small_textures)
    assert np.array_equal(st[:, :11].astype(np.float32), out["state"], equal_nan=True)
    assert np.array_equal(rgb, out["rgb"], equal_nan=True)
    assert np.array_equal(oracle.post(rgb, d.width, d.height, S, False), out["image"])


@pytest.mark.parametrize("name", ["plugin_sph_64x36_s1", "plugin_sph_32x18_s4"])
def test_plugin_fixture_is_the_reference_output(name):
    """The spherical-header fixtures are what the reference's own frame pipeline, built with
    metrics/"schwarzschild - sph.cuh" and SPHERICAL, renders from the deck (bit for bit, live,
    where the reference tree is mounted); every ray ends with SUCCESS, at the horizon or at rout."""
    from pathlib import Path

    from golden.make_golden import ALL_CASES
    from oracles import RefHost, ref_available, write_deck

    d, tex, z = load_case(name)
    st = z["state"]
    assert np.all(st[:, 2] == abi.RESULT_SUCCESS)
    r = st[:, 3]
    assert np.all((r >= 100.0) | (r <= 2.0 + 0.001 + 1e-6))
    assert 0 < np.mean(r >= 100.0) < 1
    if not ref_available("sph"):
        pytest.skip("reference host build with the spherical header not built here")
    spec = ALL_CASES[name]
    _, a_deg, b_deg = scenes.camera_pose(spec[6], spec[7])
    deck = write_deck(Path("/tmp/prrsphgolden"), d, tex, fov_deg=spec[8], a_deg=a_deg, b_deg=b_deg)
    ref = RefHost("sph")
    assert ref.load(deck) == 1
    out = ref.frame(0, fxaa=True)
    assert np.array_equal(out["state"], st, equal_nan=True)
    assert np.array_equal(out["image"], z["image"])


def test_reference_cuda_build_exports_its_driver():
    """oracle/_ref/libprr_refcu_kerr.so (the reference's own sources built with nvcc for sm_100a,
    measured by the bench beside the product) loads without a GPU and exports its driver."""
    import ctypes as C

    from oracles import REF_DIR

    p = REF_DIR / "libprr_refcu_kerr.so"
    if not p.exists():
        pytest.skip("reference CUDA build not built here")
    lib = C.CDLL(str(p))
    for name in ("prr_refcu_load", "prr_refcu_render", "prr_refcu_trace_rows", "prr_refcu_set_eps", "prr_refcu_info"):
        assert hasattr(lib, name), name
