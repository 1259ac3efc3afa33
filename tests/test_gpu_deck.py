"""The deck-driven host on the GPU: prr_run_deck and the `prr` command on a
reference-format deck (two frames, a sphere that moves between them, a mass
override) render the frames the reference renders from the same deck.

* PNG files are named <out>image_<i>.png (prr.cpp:336) and hold exactly the
  8-bit image prr_render gives for prr_deck_frame(i).
* Against the reference's own frame pipeline run on the host from the same
  deck files (oracle/_ref, frames rendered in order as prr.cpp:382-386
  does): the image is within 1/255 on >= 99.9% of pixels, the REFERENCE-mode
  image bar.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import pixel_rule, quantize
from parrelray_b200 import Deck, abi, load_image, scenes
from parrelray_b200.abi import LIB_PATH

pytestmark = pytest.mark.gpu

DECK_DIR = Path("/tmp/prrdeckgpu")  # no '_' in deck paths (main/io.h:30-36)


@pytest.fixture(scope="module")
def deck_path(small_textures):
    from oracles import write_deck

    sph = [(*scenes.orbit_point(10.0, 60.0), 1.5, scenes.SPHERE_ID0), (*scenes.orbit_point(12.0, 200.0), 2.0, 2)]
    d = scenes.make_frame(96, 54, r=30.0, incl_deg=85.0, fov_deg=60.0, metric=abi.METRIC_SCHWARZSCHILD, mass=1.0,
                          spheres=sph, mode=abi.MODE_REFERENCE, eps=1e-3, horizon_eps=0.001)
    _, a_deg, b_deg = scenes.camera_pose(30.0, 85.0)
    sim = write_deck(DECK_DIR, d, small_textures, fov_deg=60.0, a_deg=a_deg, b_deg=b_deg)
    root = sim.parent
    # frame 1: camera moved and tilted, black-hole mass 1.2 from here on;
    # sphere 0 moves in x only (y, z, r keep their frame-0 values)
    with open(root / "traj.params", "a") as f:
        f.write("_frame1_\n<x> = <28>\n<y> = <2>\n<z> = <3>\n<a> = <184>\n<b> = <-4>\n<mass> = <1.2>\n")
    with open(root / "scene.params", "a") as f:
        f.write("_sphere0_\n<x1> = <6>\n")
    return sim


def test_run_deck_writes_the_frames_prr_render_gives(gpu, small_textures, deck_path):
    deck = Deck(deck_path)
    assert deck.frame_count == 2
    out = deck_path.parent / "out"
    out.mkdir(exist_ok=True)
    st = gpu.run_deck(deck_path, prefix=str(out) + "/")
    assert st.rays == 2 * 96 * 54
    frames = [deck.frame(i) for i in range(2)]
    assert frames[1].mass == np.float32(1.2) and frames[1].spheres[0].center[0] == 6.0
    for i, f in enumerate(frames):
        png = load_image(out / f"image_{i}.png")[..., :3]
        mine = gpu.render(f)[0][0]
        assert np.array_equal(png, mine), i
    # the `prr` command writes the same files
    out2 = deck_path.parent / "cli"
    out2.mkdir(exist_ok=True)
    exe = LIB_PATH.parent / "prr"
    r = subprocess.run([str(exe), "-t", str(deck_path), "--out", str(out2) + "/"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    for i in range(2):
        assert np.array_equal(load_image(out2 / f"image_{i}.png"), load_image(out / f"image_{i}.png"))


def test_run_deck_matches_the_reference_frame_loop(gpu, small_textures, deck_path):
    from oracles import RefHost, ref_available

    if not ref_available("schw"):
        pytest.skip("reference host build (oracle/_ref) not built")
    out = deck_path.parent / "out3"
    out.mkdir(exist_ok=True)
    gpu.run_deck(deck_path, prefix=str(out) + "/")
    ref = RefHost("schw")
    assert ref.load(deck_path) == 2
    for i in range(2):  # in order: the scene update carries state from frame to frame
        z = ref.frame(i)
        png = load_image(out / f"image_{i}.png")[..., :3]
        ok = pixel_rule(png, quantize(z["image"]))
        assert ok >= 0.999, (i, ok)


def test_run_deck_reports_missing_textures(gpu, tmp_path):
    bad = DECK_DIR / "missingtex.params"
    bad.write_text("_tracer_\n<solver> = <rkf>\n<bimage1> = </nonexistent/sky.png>\n<rout1> = <100>\n<h> = <0.01>\n"
                   "<hmin> = <1e-4>\n<hmax> = <0.1>\n<eps> = <1e-3>\n_spacetime_\n<hasBlackHole> = <1>\n"
                   "<mass> = <1>\n_camera_\n<vfov> = <60>\n<width> = <8>\n<height> = <8>\n<SSAA> = <none>\n"
                   "<SSAAsamples> = <1>\n_frame0_\n<x> = <30>\n<y> = <0>\n<z> = <0>\n<a> = <180>\n<b> = <0>\n")
    with pytest.raises(abi.PrrError) as e:
        gpu.run_deck(bad, prefix=str(DECK_DIR) + "/")
    assert e.value.status == abi.ERR_IO and "sky.png" in str(e.value)


def test_deck_names_a_metric_plugin(gpu, small_textures, deck_path):
    """spacetime.metric = <a plug-in library>: the frames come from the plug-in's hooks (here the
    reference's own Schwarzschild header compiled unchanged, or the shipped Kerr header at a = 0)."""
    lib = LIB_PATH.parent / "libprr_metric_schwarzschild.so"
    if not lib.exists():
        lib = LIB_PATH.parent / "libprr_metric_kerr.so"
    # a deck value must not contain '_' (it would open a block, main/io.h:30-36): link the library
    link = deck_path.parent / "metricplugin.so"
    if not link.exists():
        link.symlink_to(lib)
    text = deck_path.read_text().replace("_spacetime_\n", f"_spacetime_\n<metric> = <{link}>\n")
    plugdeck = deck_path.parent / "plugin.params"
    plugdeck.write_text(text)
    out = deck_path.parent / "outplug"
    out.mkdir(exist_ok=True)
    gpu.run_deck(plugdeck, prefix=str(out) + "/", count=1)
    d = Deck(plugdeck)
    f = d.frame(0)
    assert f.metric == abi.METRIC_PLUGIN0
    mine = load_image(out / "image_0.png")[..., :3]
    f.metric = abi.METRIC_SCHWARZSCHILD
    ref = gpu.render(f)[0][0]
    assert pixel_rule(mine, ref) >= 0.999
