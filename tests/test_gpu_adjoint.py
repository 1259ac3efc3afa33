"""GPU discrete adjoint (prr_adjoint, reverse mode with checkpoints every 64
accepted steps) against the FP64 host gradient (forward-mode dual numbers
through the same frozen-step map) and central finite differences (h = 1e-4,
pixels with unchanged discrete events), and the torch.autograd wrapper."""
import ctypes as C
import math

import numpy as np
import pytest

from parrelray_b200 import abi, scenes
from test_oracle_gradient import NAMES, base_params, grad_frame, masked_fd

pytestmark = pytest.mark.gpu


def gpu_adjoint(gpu, d, w, sphere=0):
    g = np.zeros(5, dtype=np.float64)
    st = abi.Stats()
    wl = np.ascontiguousarray(w, dtype=np.float32)
    abi.check(abi.load().prr_adjoint(gpu.h, C.byref(d), wl.ctypes.data_as(abi._fp), sphere,
                                     g.ctypes.data_as(abi._dp), C.byref(st)), gpu.h)
    return g, st


@pytest.mark.parametrize("samples", [1, 4])
def test_adjoint_matches_host_gradient(gpu, oracle, small_textures, samples):
    d = grad_frame(W=24 if samples == 1 else 12, H_=16 if samples == 1 else 8, samples=samples, tol=1e-8)
    gpu.upload_textures(small_textures)
    w = np.random.default_rng(11).normal(size=(d.height, d.width, 3)).astype(np.float32)
    g_gpu, st = gpu_adjoint(gpu, d, w)
    g_host, _ = oracle.grad(d, small_textures, w, 0)
    assert st.n_math_error == 0 and st.accepted > 0
    for k in range(5):
        assert abs(g_gpu[k] - g_host[k]) <= 1e-5 * np.abs(g_host).max() + 1e-4 * abs(g_host[k]), (NAMES[k], g_gpu, g_host)


def test_adjoint_matches_central_differences(gpu, oracle, small_textures):
    d = grad_frame(W=16, H_=12, tol=1e-8)
    gpu.upload_textures(small_textures)
    w = np.random.default_rng(5).normal(size=(d.height, d.width, 3)).astype(np.float32)
    p0 = base_params(d)
    oracle.grad(d, small_textures, w, 0, params=p0)
    s0 = oracle.last_sig.copy()
    for k in range(5):
        fd, mask = masked_fd(oracle, d, small_textures, w, p0, k, s0)
        g, _ = gpu_adjoint(gpu, d, w * mask[:, :, None])
        assert abs(g[k] - fd) <= 1e-3 * abs(fd) + 1e-9, (NAMES[k], g[k], fd)


def smooth_sky(w=64, h=32):
    """A low-frequency sky: with it the image is a smooth function of the
    camera, so the inverse problem is well posed (a point-star sky makes the
    L2 image loss nearly random in the inclination)."""
    x = np.arange(w)[None, :]
    y = np.arange(h)[:, None]
    t = np.zeros((h, w, 4), np.uint8)
    t[..., 0] = (128 + 90 * np.sin(2 * np.pi * x / w) * np.ones_like(y)).astype(np.uint8)
    t[..., 1] = (128 + 90 * np.cos(np.pi * y / h) * np.ones_like(x)).astype(np.uint8)
    t[..., 2] = (128 + 60 * np.sin(4 * np.pi * x / w + 2 * np.pi * y / h)).astype(np.uint8)
    t[..., 3] = 255
    return t


def test_torch_wrapper_and_adam_fit(gpu, small_textures):
    import torch

    from torch_render import render

    tex = dict(small_textures)
    tex[scenes.SKY_ID] = smooth_sky()
    gpu.upload_textures(tex)
    W = H = 48
    target_p = torch.tensor([0.7, 1.0, math.radians(60.0), 20.0, math.radians(30.0)], dtype=torch.float64)
    with torch.no_grad():
        target = render(target_p, gpu, W, H)
    p = torch.tensor([0.3, 1.0, math.radians(45.0), 20.0, math.radians(30.0)], dtype=torch.float64, requires_grad=True)
    # the wrapper's gradient is prr_adjoint's
    loss = ((render(p, gpu, W, H) - target) ** 2).sum()
    loss.backward()
    d = scenes.make_frame(W, H, r=20.0, incl_deg=45.0, fov_deg=40.0, metric=abi.METRIC_KERR, spin=0.3,
                          spheres=[(*scenes.orbit_point(9.0, 30.0), 1.0, scenes.SPHERE_ID0)],
                          bg_filter=abi.BG_BILINEAR, precision=abi.PREC_FP64)
    _, img, _ = gpu.render(d, want_float=True)
    g, _ = gpu_adjoint(gpu, d, 2.0 * (img[0] - target.numpy()))
    assert np.allclose(p.grad.numpy(), g, rtol=1e-6, atol=1e-9)
    # Adam on (spin, inclination) from (0.3, 45 deg) towards (0.7, 60 deg).  The image loss is not
    # convex in (a, i): with a constant step Adam overshoots its valley (the loss falls by 45% and
    # climbs back), so the step decays by 0.95 per iteration.  Which local valley the fit settles in
    # depends on the last bits of the renders (the same fit through the FP64 CPU oracle's render and
    # gradient ends at 0.58x the start loss, a = 0.47, i = 53.3 deg; on the GPU at 0.68x), so the bars
    # are that the loss falls by a quarter and both parameters move towards the target.
    q = torch.tensor([0.3, math.radians(45.0)], dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([q], lr=0.02)
    sched = torch.optim.lr_scheduler.ExponentialLR(opt, gamma=0.95)
    losses = []
    for it in range(60):
        opt.zero_grad()
        full = torch.cat([q[:1], torch.tensor([1.0], dtype=torch.float64), q[1:],
                          torch.tensor([20.0, math.radians(30.0)], dtype=torch.float64)])
        loss = ((render(full, gpu, W, H) - target) ** 2).sum()
        loss.backward()
        opt.step()
        sched.step()
        with torch.no_grad():
            q[0].clamp_(0.0, 0.99)
        losses.append(loss.item())
    fit = (losses[::10], q[0].item(), math.degrees(q[1].item()))
    assert losses[-1] < 0.75 * losses[0], fit
    assert 0.33 < q[0].item() < 0.99, fit
    assert math.radians(46.0) < q[1].item() < math.radians(70.0), fit


def test_fp32_forward_adjoint_tracks_the_fp64_one(gpu, small_textures):
    """The differentiable-render workload's form: forward steps in FP32 (tolerance 1e-6, Kahan-
    compensated), adjoint and reduction in FP64.  Against the all-FP64 adjoint of the same frame
    and loss: the two discrete maps differ only where an FP32 step decision flips, so the gradient
    vectors agree to 2% (their norms), and each component the loss depends on strongly to 5%."""
    tex = dict(small_textures)
    tex[scenes.SKY_ID] = smooth_sky()
    gpu.upload_textures(tex)
    kw = dict(size=64, spin=0.3, incl_deg=45.0)
    _, tgt, _ = gpu.render(scenes.kerr_512_adjoint(spin=0.7, incl_deg=60.0, size=64, precision=abi.PREC_FP64),
                           want_float=True)
    d64 = scenes.kerr_512_adjoint(precision=abi.PREC_FP64, **kw)
    _, cur, _ = gpu.render(d64, want_float=True)
    dl = 2.0 * (cur[0] - tgt[0])
    g64, s64 = gpu_adjoint(gpu, d64, dl)
    g32, s32 = gpu_adjoint(gpu, scenes.kerr_512_adjoint(precision=abi.PREC_FP32, **kw), dl)
    assert s32.n_math_error == 0 and s32.accepted > 0
    assert np.linalg.norm(g32 - g64) <= 0.02 * np.linalg.norm(g64), (g32, g64)
    big = np.abs(g64) > 0.1 * np.abs(g64).max()
    assert np.all(np.abs(g32[big] - g64[big]) <= 0.05 * np.abs(g64[big])), (g32, g64)


def test_sky_weighted_adam_fit_recovers_spin_and_inclination(gpu, small_textures):
    """The differentiable-render workload's inverse problem at 128x128 (FP32 forward, FP64 adjoint,
    no sphere): Adam from (a, i) = (0.3, 45 deg) on the L2 loss over the pixels that show sky in both
    images at least 2 px from the shadow (inverse.sky_weights) reaches the target (0.7, 60 deg)."""
    from parrelray_b200 import inverse

    tex = dict(small_textures)
    tex[scenes.SKY_ID] = smooth_sky()
    gpu.upload_textures(tex)

    def frame_at(q):
        return scenes.kerr_512_adjoint(spin=float(q[0]), incl_deg=math.degrees(q[1]), precision=abi.PREC_FP32,
                                       size=128, spheres=[])

    _, tgt, _ = gpu.render(frame_at((0.7, math.radians(60.0))), want_float=True)
    h = inverse.fit(gpu, frame_at, tgt[0], (0.3, math.radians(45.0)), (0, 2), iters=150, lr=0.01, decay=0.99,
                    margin=2, lo=(0.0, 0.0), hi=(0.99, math.pi))
    a, incl = h["q_final"][0], math.degrees(h["q_final"][1])
    info = (a, incl, [round(x, 2) for x in h["loss"][::15]])
    assert abs(a - 0.7) < 0.02 and abs(incl - 60.0) < 0.3, info
    assert h["loss"][-1] < 0.01 * h["loss"][0], info


def test_adjoint_does_not_depend_on_earlier_calls(gpu, small_textures):
    """The adjoint's recomputed segments repeat its forward steps exactly (one out-of-line step
    function), so no ray is dropped as inconsistent, and an FP32-forward gradient is the same
    whether the previous call was an FP64-forward adjoint (whose checkpoints and stack are laid out
    differently) or nothing: nothing is read that the call did not write."""
    tex = dict(small_textures)
    tex[scenes.SKY_ID] = smooth_sky()
    gpu.upload_textures(tex)
    kw = dict(size=64, spin=0.3, incl_deg=45.0, spheres=[])
    _, tgt, _ = gpu.render(scenes.kerr_512_adjoint(spin=0.7, incl_deg=60.0, size=64, spheres=[]), want_float=True)
    d32 = scenes.kerr_512_adjoint(precision=abi.PREC_FP32, **kw)
    _, cur, _ = gpu.render(d32, want_float=True)
    dl = 2.0 * (cur[0] - tgt[0])
    g1, s1 = gpu.adjoint(d32, dl)
    g64, s64 = gpu.adjoint(scenes.kerr_512_adjoint(precision=abi.PREC_FP64, **kw), dl)
    g2, s2 = gpu.adjoint(d32, dl)
    for s in (s1, s64, s2):
        assert s.n_math_error == 0 and s.accepted > 0
    assert np.allclose(g1, g2, rtol=1e-9, atol=1e-9), (g1, g2)
    assert np.all(np.isfinite(g64)) and np.linalg.norm(g1 - g64) <= 0.05 * np.linalg.norm(g64), (g1, g64)
