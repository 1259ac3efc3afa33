"""The reference's own CUDA build (oracle/_ref/libprr_refcu_kerr.so: its
sources compiled with nvcc for sm_100a, measured by the bench as the
reference's GPU baseline) renders what the reference's host build renders:
its frame pipeline (prr.cpp:renderframe) on the deck of the golden Kerr case
against that case's image, which the reference host build produced
(tests/golden/kerr_48x27_s1.npz).  The reference ends its process on any CUDA
error (prr.cpp:37-47), so it runs in a child process.  nvcc contracts
multiply-adds where the host build does not, so a few rays may end
differently: >= 99% of the pixels within 1/255."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import pixel_rule, quantize
from oracles import REF_DIR, write_deck
from parrelray_b200 import scenes
from test_oracle_golden import load_case

pytestmark = pytest.mark.gpu

CHILD = r"""
import ctypes as C, sys
import numpy as np
lib = C.CDLL(sys.argv[1])
lib.prr_refcu_load.restype = C.c_int
lib.prr_refcu_load.argtypes = [C.c_char_p]
lib.prr_refcu_render.restype = C.c_double
lib.prr_refcu_render.argtypes = [C.c_int, C.POINTER(C.c_float)]
assert lib.prr_refcu_load(sys.argv[2].encode()) == 1
w, h = int(sys.argv[3]), int(sys.argv[4])
img = np.zeros((h, w, 3), dtype=np.float32)
assert lib.prr_refcu_render(0, img.ctypes.data_as(C.POINTER(C.c_float))) > 0
np.save(sys.argv[5], img)
"""


def test_reference_cuda_build_renders_the_reference_image(tmp_path):
    lib = REF_DIR / "libprr_refcu_kerr.so"
    if not lib.exists():
        pytest.skip("reference CUDA build not built (it needs the reference tree at build time)")
    d, tex, z = load_case("kerr_48x27_s1")
    _, a_deg, b_deg = scenes.camera_pose(25.0, 80.0)
    deck = write_deck(Path("/tmp/prrrefcudatest"), d, tex, fov_deg=50.0, a_deg=a_deg, b_deg=b_deg)
    out = tmp_path / "img.npy"
    r = subprocess.run([sys.executable, "-c", CHILD, str(lib), str(deck), str(d.width), str(d.height), str(out)],
                       stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    img = np.load(out)
    assert img.shape == z["image"].shape
    assert pixel_rule(quantize(img), quantize(z["image"])) >= 0.99
