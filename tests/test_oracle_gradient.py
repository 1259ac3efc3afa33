"""The FP64 host gradient (forward-mode dual numbers through the frozen-step
PHYSICAL trace, oracle/prr_oracle.cpp:prr_oracle_grad) against central finite
differences, h = 1e-4, of the same FP64 trace with the parameters perturbed
in double.

The loss is linear in the image, L = sum(w * image) with fixed random w, so
dL/dimage = w.  A gradient with frozen step sizes and events is the
derivative of the smooth part of the render; a finite difference also sees
the few pixels whose discrete outcome changes inside +-h (a ray ending one
step earlier, a ray crossing a silhouette).  Those pixels are found by the
oracle's per-pixel event signature (result and accepted-step count of every
sample) and left out of both sides.  Bar: 1e-3 relative.
"""
import numpy as np
import pytest

from parrelray_b200 import abi, scenes

NAMES = ["spin", "mass", "inclination", "camera_r", "sphere_phase"]
H = 1e-4


def grad_frame(W=20, H_=14, spin=0.7, tol=1e-8, samples=1):
    return scenes.make_frame(
        W, H_, r=20.0, incl_deg=60.0, fov_deg=40.0, metric=abi.METRIC_KERR, mass=1.0, spin=spin, samples=samples,
        spheres=[(*scenes.orbit_point(9.0, 30.0), 1.0, scenes.SPHERE_ID0)], bg_filter=abi.BG_BILINEAR,
        precision=abi.PREC_FP64, tol=tol, max_steps=200000)


def base_params(d):
    pos = np.array(d.cam_pos[:], dtype=np.float64)
    c = d.spheres[0].center
    return np.array([d.spin, d.mass, np.arccos(pos[2] / np.linalg.norm(pos)), np.linalg.norm(pos),
                     np.arctan2(c[1], c[0])], dtype=np.float64)


def masked_fd(oracle, d, tex, w, p0, k, s0, h=H):
    """Central difference of sum(w*image) (FP64 images) over pixels whose
    discrete events are the same at p0-h, p0 and p0+h; returns (fd, mask)."""
    pp, pm = p0.copy(), p0.copy()
    pp[k] += h
    pm[k] -= h
    _, ip = oracle.grad(d, tex, w, 0, params=pp)
    sp = oracle.last_sig.copy()
    _, im = oracle.grad(d, tex, w, 0, params=pm)
    sm = oracle.last_sig.copy()
    mask = (s0 == sp) & (s0 == sm)
    wm = w.astype(np.float64) * mask[:, :, None]
    return (np.sum(wm * ip) - np.sum(wm * im)) / (2 * h), mask


@pytest.mark.parametrize("samples", [1, 4])
def test_host_gradient_matches_central_differences(oracle, small_textures, samples):
    d = grad_frame(samples=samples, W=10 if samples == 4 else 16, H_=8 if samples == 4 else 12)
    w = np.random.default_rng(5).normal(size=(d.height, d.width, 3)).astype(np.float32)
    p0 = base_params(d)
    st, _ = oracle.trace(d, small_textures, precision=1)
    assert (st[:, 2] == abi.RESULT_INTERSECTION).sum() > 0  # the sphere is in view
    oracle.grad(d, small_textures, w, 0, params=p0)
    s0 = oracle.last_sig.copy()
    for k in range(5):
        fd, mask = masked_fd(oracle, d, small_textures, w, p0, k, s0)
        # pixels of 4 samples change events more often (any sample may)
        assert mask.mean() > (0.8 if samples == 1 else 0.5), (NAMES[k], mask.mean())
        g, _ = oracle.grad(d, small_textures, w * mask[:, :, None], 0, params=p0)
        assert abs(g[k] - fd) <= 1e-3 * abs(fd) + 1e-9, (NAMES[k], g[k], fd)
