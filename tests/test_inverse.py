"""The inverse-problem helpers on the host: the sky weights, the Adam update
and the fit loop's plumbing (with a stand-in renderer whose gradient is known)."""
import math

import numpy as np
import pytest

from parrelray_b200 import inverse


def brute_weights(image, target, margin):
    sky = (image.max(axis=2) > 0) & (target.max(axis=2) > 0)
    h, w = sky.shape
    out = np.zeros((h, w), np.float32)
    for y in range(h):
        for x in range(w):
            ok = True
            for yy in range(y - margin, y + margin + 1):
                for xx in range(x - margin, x + margin + 1):
                    if 0 <= yy < h and 0 <= xx < w and not sky[yy, xx]:
                        ok = False
            out[y, x] = ok
    return out


@pytest.mark.parametrize("margin", [0, 1, 2, 3])
def test_sky_weights_match_a_brute_force_erosion(margin):
    rng = np.random.default_rng(margin)
    img = rng.uniform(0.1, 1.0, (23, 31, 3))
    tgt = rng.uniform(0.1, 1.0, (23, 31, 3))
    yy, xx = np.mgrid[:23, :31]
    img[(yy - 11) ** 2 + (xx - 12) ** 2 < 30] = 0.0   # a shadow
    tgt[(yy - 9) ** 2 + (xx - 17) ** 2 < 20] = 0.0
    img[0, 30] = 0.0                                  # a black pixel on the border
    tgt[22, :3] = (0.0, 0.0, 0.0)
    w = inverse.sky_weights(img, tgt, margin)
    assert w.dtype == np.float32 and w.shape == (23, 31)
    assert np.array_equal(w, brute_weights(img, tgt, margin))


def test_sky_weights_treat_one_lit_channel_as_sky_and_reject_bad_shapes():
    img = np.zeros((4, 4, 3))
    img[..., 2] = 0.5
    assert inverse.sky_weights(img, img, 1).all()
    with pytest.raises(ValueError):
        inverse.sky_weights(img, img[:3], 1)
    with pytest.raises(ValueError):
        inverse.sky_weights(img, img, -1)


def test_adam_first_step_is_lr_along_the_gradient_sign_and_clips():
    opt = inverse.Adam([1.0, 2.0], lr=0.1, lo=[0.0, 0.0], hi=[1.05, 5.0])
    q = opt.step([-3.0, 0.5])
    assert np.allclose(q, [1.05, 1.9], atol=1e-6)  # +0.1 clipped at 1.05; -0.1
    q = inverse.Adam([0.0], lr=0.05, decay=0.5).step([1e-3])
    assert np.allclose(q, [-0.05], atol=1e-6)


def test_adam_minimises_a_quadratic():
    target = np.array([0.7, -0.3])
    opt = inverse.Adam([0.3, 0.8], lr=0.05, decay=0.99)
    for _ in range(300):
        opt.step(2.0 * (opt.q - target))
    assert np.allclose(opt.q, target, atol=2e-3)


class FakeCtx:
    """Renders image(q) = q0 A + q2 B (inside a fixed black disc: 0) and
    returns the exact adjoint of that linear map."""

    class St:
        kernel_ms = 1.0
        trace_ms = 2.0

    def __init__(self):
        rng = np.random.default_rng(7)
        self.A = rng.uniform(0.2, 1.0, (16, 16, 3))
        self.B = rng.uniform(0.2, 1.0, (16, 16, 3))
        yy, xx = np.mgrid[:16, :16]
        self.hole = ((yy - 8) ** 2 + (xx - 8) ** 2 < 9)[:, :, None]
        self.seen_weights = []

    def image(self, q):
        return np.where(self.hole, 0.0, q[0] * self.A + q[2] * self.B)

    def render(self, d, want_float=False):
        return None, [self.image(d).astype(np.float32)], self.St()

    def adjoint(self, d, dl, sphere_index=-1):
        self.seen_weights.append(dl)
        g = np.zeros(5)
        g[0] = np.sum(dl * np.where(self.hole, 0.0, self.A))
        g[2] = np.sum(dl * np.where(self.hole, 0.0, self.B))
        return g, self.St()


def test_fit_loop_converges_with_the_weighted_loss_and_reports_its_history():
    ctx = FakeCtx()
    q_true = np.array([0.7, 0.0, 1.2, 0.0, 0.0])

    def frame_at(q):
        return np.array([q[0], 0.0, q[1], 0.0, 0.0])

    target = ctx.image(q_true)
    h = inverse.fit(ctx, frame_at, target, (0.3, 0.8), (0, 2), iters=400, lr=0.02, decay=0.995, margin=1)
    assert np.allclose(h["q_final"], [0.7, 1.2], atol=5e-3)
    assert len(h["loss"]) == 400 and h["loss"][-1] < 1e-3 * h["loss"][0]
    assert all(ms == 4.0 for ms in h["device_ms"])  # render 1 + adjoint 1 + its forward 2
    # the dL/dimage the adjoint received is zero on the shadow and its 1-pixel rim
    w = inverse.sky_weights(ctx.image(frame_at((0.3, 0.8))), target, 1)
    assert np.all(ctx.seen_weights[0][w == 0] == 0.0)
    assert 0 < h["weighted_fraction"][0] < 1 and math.isclose(h["weighted_fraction"][0], float(w.mean()))
