"""Generates tests/golden/*.npz from the REFERENCE ITSELF: the reference's
sources compiled for the host (oracle/_ref, built by oracle/ref/build_ref.sh
from the reference tree) run through reference-format decks written here.

    python tests/golden/make_golden.py

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

# name: (metric tag, metric, W, H, S, spin, r, incl, fov, eps, spheres (orbit, phase, radius, tex))
CASES = {
    "schw_160x90_s1": ("schw", abi.METRIC_SCHWARZSCHILD, 160, 90, 1, 0.0, 30.0, 85.0, 60.0, 1e-3,
                       [(10.0, 60.0, 1.5, 1), (12.0, 200.0, 2.0, 2)]),
    "schw_64x36_s4": ("schw", abi.METRIC_SCHWARZSCHILD, 64, 36, 4, 0.0, 25.0, 80.0, 50.0, 1e-4,
                      [(8.0, 35.0, 1.0, 1), (14.0, 300.0, 1.2, 2), (6.5, 160.0, 0.5, 3)]),
    "flat_64x36_s1": ("flat", abi.METRIC_FLAT, 64, 36, 1, 0.0, 30.0, 70.0, 60.0, 1e-3,
                      [(10.0, 10.0, 3.0, 1)]),
    "kerr_48x27_s1": ("kerr", abi.METRIC_KERR, 48, 27, 1, 0.9, 25.0, 80.0, 50.0, 1e-3,
                      [(9.0, 40.0, 1.0, 1)]),
}

# Metric plug-in headers of the reference run through its own frame pipeline
# (files named plugin_*): the reference's spherical-coordinate Schwarzschild
# header metrics/"schwarzschild - sph.cuh", built with SPHERICAL.  It ignores
# the scene's spheres, so these frames have none.
PLUGIN_CASES = {
    "plugin_sph_64x36_s1": ("sph", abi.METRIC_SCHWARZSCHILD, 64, 36, 1, 0.0, 30.0, 85.0, 60.0, 1e-3, []),
    "plugin_sph_32x18_s4": ("sph", abi.METRIC_SCHWARZSCHILD, 32, 18, 4, 0.0, 20.0, 88.0, 50.0, 1e-4, []),
}
ALL_CASES = {**CASES, **PLUGIN_CASES}

SKY = (256, 128)
SPH = (128, 64)


def textures():
    tex = {scenes.SKY_ID: scenes.make_texture(1, 1234, *SKY)}
    for k in range(3):
        tex[scenes.SPHERE_ID0 + k] = scenes.make_texture(0, 100 + k, *SPH)
    return tex


def texture_digest(tex) -> str:
    h = hashlib.sha256()
    for k in sorted(tex):
        h.update(np.ascontiguousarray(tex[k]).tobytes())
    return h.hexdigest()


def case_frame(spec) -> tuple[abi.FrameDesc, dict]:
    tag, metric, W, H, S, spin, r, inc, fov, eps, sph = spec
    spheres = [(*scenes.orbit_point(orb, ph), rad, tex) for (orb, ph, rad, tex) in sph]
    d = scenes.make_frame(W, H, r=r, incl_deg=inc, fov_deg=fov, metric=metric, mass=1.0, spin=spin, samples=S,
                          mode=abi.MODE_REFERENCE, eps=eps, horizon_eps=0.001, rout=100.0, spheres=spheres)
    meta = dict(tag=tag, metric=metric, W=W, H=H, S=S, spin=spin, r=r, incl=inc, fov=fov, eps=eps,
                spheres=[list(s) for s in sph])
    return d, meta


def main() -> int:
    build.build_library()
    if not build.build_reference():
        print("reference tree not found; cannot regenerate golden fixtures", file=sys.stderr)
        return 2
    tex = textures()
    digest = texture_digest(tex)
    for name, spec in ALL_CASES.items():
        d, meta = case_frame(spec)
        _, a_deg, b_deg = scenes.camera_pose(spec[6], spec[7])
        deck = write_deck(Path("/tmp/prrgolden"), d, tex, fov_deg=spec[8], a_deg=a_deg, b_deg=b_deg)
        ref = RefHost(spec[0])
        assert ref.load(deck) == 1
        out = ref.frame(0, fxaa=True)
        meta["texture_sha256"] = digest
        np.savez_compressed(HERE / f"{name}.npz", state=out["state"], rgb=out["rgb"], image=out["image"],
                            fxaa=out["fxaa"], meta=json.dumps(meta))
        res = np.bincount(out["state"][:, 2].astype(int), minlength=5)
        print(f"{name}: results {res.tolist()}  {out['seconds']:.2f}s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
