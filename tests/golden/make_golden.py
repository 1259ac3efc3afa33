"""Generates tests/golden/*.npz from the REFERENCE ITSELF: the reference's
sources compiled for the host (oracle/_ref, built by oracle/ref/build_ref.sh
from the reference tree) run through reference-format decks written here.

    python tests/golden/make_golden.py [case ...]

Each case stores the frame descriptor fields needed to rebuild the same
prr_frame_desc without the reference, a checksum of the seeded textures, and
the reference outputs: per-ray state after trace_RKF (uv, result, r, u), the
per-sample colour after rayToRGB, the combineSamples image and the FXAA image
(FXAA run on the combined image; border pixels the kernel never writes are
zero).  The GPU box has no reference tree; tests there read these files.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))

from parrelray_b200 import abi, build, scenes  # noqa: E402
from oracles import RefHost, write_deck  # noqa: E402

# name: (metric tag, metric, W, H, S, spin, r, incl, fov, eps, spheres (orbit, phase, radius, tex)[, extras])
# extras: "solver" ("rkf" by default, "euler" = trace_Euler, kernels/solver.cuh:68-116) and
# "textures" ("small" by default, "standard" = the workloads' 512x256 sphere / 2048x1024 sky sizes)
CASES = {
    "schw_160x90_s1": ("schw", abi.METRIC_SCHWARZSCHILD, 160, 90, 1, 0.0, 30.0, 85.0, 60.0, 1e-3,
                       [(10.0, 60.0, 1.5, 1), (12.0, 200.0, 2.0, 2)]),
    "schw_64x36_s4": ("schw", abi.METRIC_SCHWARZSCHILD, 64, 36, 4, 0.0, 25.0, 80.0, 50.0, 1e-4,
                      [(8.0, 35.0, 1.0, 1), (14.0, 300.0, 1.2, 2), (6.5, 160.0, 0.5, 3)]),
    "flat_64x36_s1": ("flat", abi.METRIC_FLAT, 64, 36, 1, 0.0, 30.0, 70.0, 60.0, 1e-3,
                      [(10.0, 10.0, 3.0, 1)]),
    "kerr_48x27_s1": ("kerr", abi.METRIC_KERR, 48, 27, 1, 0.9, 25.0, 80.0, 50.0, 1e-3,
                      [(9.0, 40.0, 1.0, 1)]),
    # trace_Euler (prr.cpp:295-299): fixed step h = 0.01, affine length < 5000
    "euler_64x36_s1": ("schw", abi.METRIC_SCHWARZSCHILD, 64, 36, 1, 0.0, 30.0, 85.0, 60.0, 1e-3,
                       [(10.0, 60.0, 1.5, 1), (12.0, 200.0, 2.0, 2)], {"solver": "euler"}),
}

# The single-frame Schwarzschild workload at its full size (M = 1, camera r = 30M, inclination 85
# deg, FOV 60 deg, 320x180, no SSAA, one sphere R = 1M on the orbit r = 10M, the 512x256 sphere
# texture and the 2048x1024 starfield) in the reference's own solver at the two tolerances where
# its FP32 absolute error test still works.  Stored slim (files named full_*): per ray the result,
# the final direction of motion quantised to 16-bit angles, and the colour quantised to 8 bits.
FULL_CASES = {
    "full_schw_320x180_eps1e-3": ("schw", abi.METRIC_SCHWARZSCHILD, 320, 180, 1, 0.0, 30.0, 85.0, 60.0, 1e-3,
                                  [(10.0, 60.0, 1.0, 1)], {"textures": "standard"}),
    "full_schw_320x180_eps1e-4": ("schw", abi.METRIC_SCHWARZSCHILD, 320, 180, 1, 0.0, 30.0, 85.0, 60.0, 1e-4,
                                  [(10.0, 60.0, 1.0, 1)], {"textures": "standard"}),
}

# Metric plug-in headers of the reference run through its own frame pipeline
# (files named plugin_*): the reference's spherical-coordinate Schwarzschild
# header metrics/"schwarzschild - sph.cuh", built with SPHERICAL.  It ignores
# the scene's spheres, so these frames have none.
PLUGIN_CASES = {
    "plugin_sph_64x36_s1": ("sph", abi.METRIC_SCHWARZSCHILD, 64, 36, 1, 0.0, 30.0, 85.0, 60.0, 1e-3, []),
    "plugin_sph_32x18_s4": ("sph", abi.METRIC_SCHWARZSCHILD, 32, 18, 4, 0.0, 20.0, 88.0, 50.0, 1e-4, []),
}
ALL_CASES = {**CASES, **PLUGIN_CASES, **FULL_CASES}

SKY = (256, 128)
SPH = (128, 64)


def extras(spec) -> dict:
    return spec[11] if len(spec) > 11 else {}


def textures(kind: str = "small"):
    """The seeded textures of a case: "small" (256x128 sky, 128x64 spheres) or "standard"."""
    if kind == "standard":
        return scenes.standard_textures()
    tex = {scenes.SKY_ID: scenes.make_texture(1, 1234, *SKY)}
    for k in range(3):
        tex[scenes.SPHERE_ID0 + k] = scenes.make_texture(0, 100 + k, *SPH)
    return tex


def case_textures(spec):
    return textures(extras(spec).get("textures", "small"))


def quantise_direction(u: np.ndarray) -> np.ndarray:
    """Direction of the spatial vectors u (n x 3) as 16-bit polar and azimuthal angles (n x 2):
    theta in [0, pi] and phi in [-pi, pi] mapped onto 0..65535 (steps of 4.8e-5 and 9.6e-5 rad)."""
    u = u.astype(np.float64)
    n = np.linalg.norm(u, axis=1)
    n[n == 0] = 1.0
    th = np.arccos(np.clip(u[:, 2] / n, -1.0, 1.0))
    ph = np.arctan2(u[:, 1], u[:, 0])
    return np.stack([np.rint(th / np.pi * 65535.0), np.rint((ph + np.pi) / (2 * np.pi) * 65535.0)], 1).astype(np.uint16)


def dequantise_direction(q: np.ndarray) -> np.ndarray:
    th = q[:, 0].astype(np.float64) / 65535.0 * np.pi
    ph = q[:, 1].astype(np.float64) / 65535.0 * 2 * np.pi - np.pi
    return np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)


def quantise_colour(rgb: np.ndarray) -> np.ndarray:
    """roundf(255 x) of the clamped colour (cudamaths/image.cu:31)."""
    v = np.float32(255.0) * np.clip(rgb.astype(np.float32), np.float32(0.0), np.float32(1.0))
    return np.floor(v.astype(np.float64) + 0.5).astype(np.uint8)


def slim(state: np.ndarray, rgb: np.ndarray) -> dict:
    """The stored form of a full_* case."""
    return {"result": state[:, 2].astype(np.int8), "direction": quantise_direction(state[:, 7:10]),
            "rgb8": quantise_colour(rgb)}


def texture_digest(tex) -> str:
    h = hashlib.sha256()
    for k in sorted(tex):
        h.update(np.ascontiguousarray(tex[k]).tobytes())
    return h.hexdigest()


def case_frame(spec) -> tuple[abi.FrameDesc, dict]:
    tag, metric, W, H, S, spin, r, inc, fov, eps, sph = spec[:11]
    spheres = [(*scenes.orbit_point(orb, ph), rad, tex) for (orb, ph, rad, tex) in sph]
    d = scenes.make_frame(W, H, r=r, incl_deg=inc, fov_deg=fov, metric=metric, mass=1.0, spin=spin, samples=S,
                          mode=abi.MODE_REFERENCE, eps=eps, horizon_eps=0.001, rout=100.0, spheres=spheres)
    ex = extras(spec)
    if ex.get("solver") == "euler":
        d.solver = abi.SOLVER_EULER
    meta = dict(tag=tag, metric=metric, W=W, H=H, S=S, spin=spin, r=r, incl=inc, fov=fov, eps=eps,
                spheres=[list(s) for s in sph], **ex)
    return d, meta


def main() -> int:
    build.build_library()
    if not build.build_reference():
        print("reference tree not found; cannot regenerate golden fixtures", file=sys.stderr)
        return 2
    only = set(sys.argv[1:])
    for name, spec in ALL_CASES.items():
        if only and name not in only:
            continue
        tex = case_textures(spec)
        d, meta = case_frame(spec)
        _, a_deg, b_deg = scenes.camera_pose(spec[6], spec[7])
        deck = write_deck(Path("/tmp/prrgolden"), d, tex, fov_deg=spec[8], a_deg=a_deg, b_deg=b_deg,
                          solver=extras(spec).get("solver", "rkf"))
        ref = RefHost(spec[0])
        assert ref.load(deck) == 1
        out = ref.frame(0, fxaa=True)
        meta["texture_sha256"] = texture_digest(tex)
        if name in FULL_CASES:
            np.savez_compressed(HERE / f"{name}.npz", meta=json.dumps(meta), **slim(out["state"], out["rgb"]))
        else:
            np.savez_compressed(HERE / f"{name}.npz", state=out["state"], rgb=out["rgb"], image=out["image"],
                                fxaa=out["fxaa"], meta=json.dumps(meta))
        res = np.bincount(out["state"][:, 2].astype(int), minlength=5)
        print(f"{name}: results {res.tolist()}  {out['seconds']:.2f}s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
