"""The deck reader (prr_deck_*) against the reference's own parser, and the
frame descriptors it builds.  No GPU needed.

* tests/golden/decks.json holds what the reference's readParams / par / pari
  / parf / headerExists / parExists / checkFrame return on decks that
  exercise the parse quirks (tests/golden/make_deck_golden.py, run against
  the reference host build); the product must return the same, bit for bit.
* Where the reference host build is present, random decks are compared live.
* prr_deck_frame reproduces the frame a reference-format deck describes
  (camera angles converted as the reference converts them; the scene update
  rule keeps a sphere's previous value when a frame key is absent; the frame
  mass override carries over).
"""
import json
import math
import random
from pathlib import Path

import numpy as np
import pytest

from parrelray_b200 import Deck, PrrError, abi, build, scenes

GOLDEN = Path(__file__).resolve().parent / "golden" / "decks.json"
_REF = build.reference_tree()
REF_INPUT = _REF / "input" if _REF else Path("/nonexistent")


def _f(x):
    return x if not isinstance(x, str) else float(x)


def _same_float(a, b):
    a, b = float(np.float32(a)), float(np.float32(_f(b)))
    return (math.isnan(a) and math.isnan(b)) or a == b


def check_against(deck: Deck, res: dict):
    for q in res["queries"]:
        blk, key = q["block"], q["key"]
        assert deck.has(blk, key) == bool(q["has"]), (blk, key)
        assert deck.get(blk, key) == q["par"], (blk, key)
        assert deck.geti(blk, key) == q["pari"], (blk, key)
        assert _same_float(deck.getf(blk, key), q["parf"]), (blk, key, deck.getf(blk, key), q["parf"])
        assert _same_float(deck.getf(blk, key, 7.5), q["parf_default"]), (blk, key)
    for blk, has in res["has_block"].items():
        assert deck.has_block(blk) == bool(has), blk
    for blk, key, val in res["entries"]:
        assert deck.has(blk, key) and deck.get(blk, key) == val, (blk, key, val)
    assert deck.frame_count == res["check_frame"]


@pytest.mark.parametrize("name", ["quirks", "crlf_frames"])
def test_parser_matches_reference_golden(built, name):
    g = json.loads(GOLDEN.read_text())
    check_against(Deck(text=g["decks"][name]), g["results"][name])


def test_parser_matches_reference_on_a_deck_file(built, tmp_path):
    g = json.loads(GOLDEN.read_text())
    p = tmp_path / "deck.params"
    p.write_bytes(g["decks"]["crlf_frames"].encode())
    check_against(Deck(p), g["results"]["crlf_frames"])


@pytest.mark.skipif(not REF_INPUT.exists(), reason="the reference's example decks are not mounted")
@pytest.mark.parametrize("stem", ["sim", "scene", "traj"])
def test_parser_matches_reference_on_its_example_decks(built, stem):
    g = json.loads(GOLDEN.read_text())
    res = g["results"]["reference_" + stem]
    text = (REF_INPUT / f"{stem}.params").read_text(encoding="utf-8", errors="surrogateescape")
    d = Deck(text=text)
    for blk, key, val in res["entries"]:
        assert d.get(blk, key) == val, (blk, key)
    for q in res["queries"]:
        assert d.get(q["block"], q["key"]) == q["par"]


def _random_deck(rng: random.Random) -> str:
    atoms = ["_", "<", ">", "=", " ", "\t", "#", "a", "b", "x", "1", "2.5", "-", "e", "frame0", "sphere0", "\r"]
    lines = []
    for _ in range(rng.randint(5, 40)):
        kind = rng.random()
        if kind < 0.15:
            lines.append("_" + rng.choice(["tracer", "camera", "frame0", "frame1", "sphere0", "a_b"]) + "_")
        elif kind < 0.7:
            k = rng.choice(["x", "y", "z", "a", "b", "mass", "h", "key"])
            v = rng.choice(["1", "2.5", "-3e2", "abc", "0x1f", "", " 4 ", "inf", "1e99"])
            lines.append(f"<{k}> = <{v}>" + rng.choice(["", "  #c", "\r"]))
        else:
            lines.append("".join(rng.choice(atoms) for _ in range(rng.randint(0, 12))))
    return "\n".join(lines) + "\n"


def test_parser_matches_reference_live_on_random_decks(built, tmp_path):
    from oracles import ref_available

    if not ref_available("schw"):
        pytest.skip("reference host build (oracle/_ref) not built")
    import sys

    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    from make_deck_golden import RefParser

    rp = RefParser()
    rng = random.Random(5)
    for _ in range(60):
        text = _random_deck(rng)
        res = rp.table(text)
        d = Deck(text=text)
        for blk, key, val in res["entries"]:
            assert d.get(blk, key) == val, (text, blk, key)
        n_ours = sum(1 for blk, key, _ in res["entries"] if d.has(blk, key))
        assert n_ours == len(res["entries"])
        assert d.frame_count == res["check_frame"], text


def test_frame_descriptor_from_a_reference_deck(built, tmp_path, small_textures):
    """write_deck (the decks the golden fixtures were rendered from) -> the
    same descriptor the tests build directly."""
    from oracles import write_deck

    sph = [(*scenes.orbit_point(10.0, 60.0), 1.5, scenes.SPHERE_ID0), (*scenes.orbit_point(12.0, 200.0), 2.0, 2)]
    d = scenes.make_frame(160, 90, r=30.0, incl_deg=85.0, fov_deg=60.0, metric=abi.METRIC_SCHWARZSCHILD, mass=1.0,
                          spheres=sph, mode=abi.MODE_REFERENCE, eps=1e-3, horizon_eps=0.001, samples=4)
    _, a_deg, b_deg = scenes.camera_pose(30.0, 85.0)
    # deck paths must not contain '_' (it opens a block, main/io.h:30-36)
    deck_path = write_deck(Path("/tmp/prrdecktests"), d, small_textures, fov_deg=60.0, a_deg=a_deg, b_deg=b_deg)
    deck = Deck(deck_path)
    assert deck.frame_count == 1 and deck.sphere_count == 2
    f = deck.frame(0)
    for name in ("width", "height", "ssaa", "samples", "vfov", "cam_alpha", "cam_beta", "metric", "mass", "spin",
                 "solver", "mode", "precision", "h", "hmin", "hmax", "eps", "rout", "horizon_eps", "background_id",
                 "nspheres", "fxaa"):
        assert getattr(f, name) == getattr(d, name), name
    assert list(f.cam_pos) == list(d.cam_pos)
    for k in range(2):
        assert list(f.spheres[k].center) == list(d.spheres[k].center)
        assert f.spheres[k].radius == d.spheres[k].radius
    assert f.spheres[0].texture_id == 1 and f.spheres[1].texture_id == 2


def test_scene_update_rule_and_mass_override(built):
    g = json.loads(GOLDEN.read_text())
    deck = Deck(text=g["decks"]["crlf_frames"].replace("_tracer_", "_tracer_\r\n<rout1> = <100>\r\n<hmin> = <1e-4>"
                                                                    "\r\n<hmax> = <0.1>\r\n<eps> = <1e-3>")
                + "_spacetime_\n<hasBlackHole> = <1>\n<mass> = <1>\n_camera_\n<vfov> = <60>\n<SSAA> = <none>\n"
                  "<SSAAsamples> = <1>\n")
    assert deck.frame_count == 3 and deck.sphere_count == 2  # sphere3 without sphere2 is not a sphere
    f0, f1, f2 = (deck.frame(i) for i in range(3))
    # sphere0: x0=10 r0=1; frame 1 sets x1=9 (kept after), frame 2 sets r2=1.5
    assert (f0.spheres[0].center[0], f0.spheres[0].radius) == (10.0, 1.0)
    assert (f1.spheres[0].center[0], f1.spheres[0].radius) == (9.0, 1.0)
    assert (f2.spheres[0].center[0], f2.spheres[0].radius) == (9.0, 1.5)
    assert list(f2.spheres[1].center) == [-10.0, 5.0, 1.0]
    # frame1.mass = 2 overrides from frame 1 on (prr.cpp:253 keeps the last value)
    assert (f0.mass, f1.mass, f2.mass) == (1.0, 2.0, 2.0)
    assert f0.solver == abi.SOLVER_EULER and f0.ssaa == abi.SSAA_NONE
    # camera angles: float(deg * M_PI / 180.0f) as prr.cpp:246-247
    assert f1.cam_alpha == np.float32(np.float64(np.float32(181.0)) * math.pi / np.float64(np.float32(180.0)))
    assert f1.cam_beta == scenes.deg_to_rad_f32(-11.0)
    assert list(f1.cam_pos) == [24.0, 1.0, 4.0]
    with pytest.raises(PrrError):
        deck.frame(3)  # frame3 is missing, so the deck has three frames


def test_deck_options_and_unsupported_choices(built):
    base = ("_tracer_\n<solver> = <{solver}>\n<h> = <0.01>\n<hmin> = <1e-4>\n<hmax> = <0.1>\n<eps> = <1e-3>\n"
            "<rout1> = <100>\n{extra}_spacetime\n<hasBlackHole> = <{bh}>\n<mass> = <1>\n<spin> = <0.5>\n{metric}"
            "_camera_\n<vfov> = <60>\n<width> = <8>\n<height> = <8>\n<SSAA> = <{ssaa}>\n<SSAAsamples> = <{s}>\n"
            "_frame0_\n<x> = <30>\n<y> = <0>\n<z> = <0>\n<a> = <180>\n<b> = <0>\n")

    def frame(**kw):
        args = dict(solver="rkf", extra="", bh=1, metric="", ssaa="regular", s=4)
        args.update(kw)
        return Deck(text=base.format(**args)).frame(0)

    f = frame()
    assert f.mode == abi.MODE_REFERENCE and f.metric == abi.METRIC_SCHWARZSCHILD and f.samples == 4
    assert f.horizon_eps == pytest.approx(1e-3) and f.rtol == f.eps
    f = frame(metric="<metric> = <kerr>\n", extra="<mode> = <physical>\n<precision> = <split>\n<rtol> = <1e-7>\n"
                                                   "<maxsteps> = <500>\n<fxaa> = <1>\n<bgfilter> = <bilinear>\n")
    assert (f.metric, f.mode, f.precision, f.max_steps, f.fxaa, f.bg_filter) == (
        abi.METRIC_KERR, abi.MODE_PHYSICAL, abi.PREC_SPLIT, 500, 1, abi.BG_BILINEAR)
    assert f.spin == np.float32(0.5) and f.rtol == np.float32(1e-7)
    assert frame(bh=0).metric == abi.METRIC_FLAT
    assert frame(metric="<metric> = </opt/metrics/libmymetric.so>\n").metric == abi.METRIC_PLUGIN0
    assert frame(solver="nonsense").solver == abi.SOLVER_EULER       # Parameters::getSolver fallback
    assert frame(ssaa="nonsense").ssaa == abi.SSAA_REGULAR           # Parameters::getSSAA fallback
    assert frame(ssaa="jittered").ssaa == abi.SSAA_JITTERED and frame(ssaa="random").ssaa == abi.SSAA_RANDOM
    assert frame(extra="").camera == abi.CAMERA_SPHERICAL
    for bad in (dict(solver="rk"), dict(ssaa="poisson")):
        with pytest.raises(PrrError) as e:
            frame(**bad)
        assert e.value.status == abi.ERR_UNSUPPORTED
    with pytest.raises(PrrError) as e:
        frame(metric="<metric> = <reissner>\n")
    assert e.value.status == abi.ERR_INVALID


def test_deck_emission_keys(built):
    """spacetime.emission (none, disk) and the emis* keys fill prr_emission_desc; grid takes its plasma from
    prr_upload_plasma, so a deck asking for it is unsupported."""
    base = ("_tracer_\n<solver> = <rkf>\n<mode> = <physical>\n<rout1> = <100>\n<h> = <0.01>\n<hmin> = <1e-4>\n"
            "<hmax> = <0.1>\n<eps> = <1e-6>\n_spacetime_\n<hasBlackHole> = <1>\n<mass> = <1>\n<metric> = <kerr>\n"
            "<spin> = <0.9>\n{emis}_camera_\n<vfov> = <30>\n<width> = <8>\n<height> = <8>\n<SSAA> = <none>\n"
            "<SSAAsamples> = <1>\n_frame0_\n<x> = <50>\n<y> = <0>\n<z> = <0>\n<a> = <180>\n<b> = <0>\n")
    f = Deck(text=base.format(emis="")).frame(0)
    assert f.emission == abi.EMISSION_NONE
    f = Deck(text=base.format(emis="<emission> = <disk>\n<emisIndex> = <3>\n<emisHeight> = <0.25>\n"
                                   "<emisRin> = <1.5>\n<emisRout> = <25>\n<emisAlpha> = <0.7>\n<emisAbsorb> = <0.1>\n"
                                   "<emisGain> = <4>\n<emisSense> = <-1>\n<emisMap> = <grey>\n")).frame(0)
    e = f.emis
    assert f.emission == abi.EMISSION_DISK
    assert (e.index, e.height, e.r_in, e.r_out) == (3.0, np.float32(0.25), 1.5, 25.0)
    assert (e.spectral_index, e.absorb, e.gain, e.sense, e.colormap) == (
        np.float32(0.7), np.float32(0.1), 4.0, -1, abi.CMAP_GREY)
    f = Deck(text=base.format(emis="<emission> = <disk>\n")).frame(0)  # defaults of prr_frame_desc_defaults
    assert (f.emis.index, f.emis.sense, f.emis.colormap, f.emis.gain) == (2.0, 1, abi.CMAP_AFMHOT, 1.0)
    with pytest.raises(PrrError) as e:
        Deck(text=base.format(emis="<emission> = <grid>\n")).frame(0)
    assert e.value.status == abi.ERR_UNSUPPORTED
    for bad in ("<emission> = <plasma>\n", "<emission> = <disk>\n<emisMap> = <viridis>\n"):
        with pytest.raises(PrrError) as e:
            Deck(text=base.format(emis=bad)).frame(0)
        assert e.value.status == abi.ERR_INVALID


def test_missing_deck_file_is_an_io_error(built, tmp_path):
    with pytest.raises(PrrError) as e:
        Deck(tmp_path / "nope.params")
    assert e.value.status == abi.ERR_IO
