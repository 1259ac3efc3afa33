"""Known-answer tests of the CPU restatement's plasma emission (the model of
prr_emission in include/prr.h; the reference declares the plasma fields,
main/Spacetime.h:50-51, and the luminosity Ray::I, main/base.h:175, without
using them, so the oracle is pinned by analytic answers):

* flat space, uniform static plasma: I is the chord length through the
  emitting shell; with grey absorption kappa, I = (1 - exp(-kappa L))/kappa
  and the transmittance is exp(-kappa L);
* flat space, uniform flow v: the Doppler factor g = 1 / (gamma (1 - v.n))
  of the traced direction n, I = g^(2 + alpha) L, optical depth kappa L / g;
* a plasma grid that is linear in x, y, z is reproduced exactly by the
  trilinear interpolation: I is the line integral of the linear density
  (times Theta^temp_power);
* Schwarzschild, static plasma on a radial ray: gravitational redshift
  g = sqrt((1 - 2M/r) / (1 - 2M/r_cam)) and dr/dlambda = -E give
  I = (r2 - r1 - 2M ln(r2/r1)) / (1 - 2M/r_cam)^(3/2);
* a Keplerian disk seen edge-on in Schwarzschild: reversing the flow mirrors
  the image, and the image is not mirror-symmetric (Doppler beaming).
"""
import math

import numpy as np
import pytest

from parrelray_b200 import abi, scenes


def flat_frame(w=1, h=1, fov_deg=10.0, hmax=0.01, r=30.0):
    d = scenes.make_frame(w, h, r=r, incl_deg=90.0, fov_deg=fov_deg, metric=abi.METRIC_FLAT, precision=abi.PREC_FP64,
                          background=False, hmax=hmax, tol=1e-9, max_steps=200000)
    return d


def shell_segments(cam, n, r_in, r_out):
    """Parameter intervals [s1, s2] of the line cam + s n (s > 0) with r_in <= |x| <= r_out."""
    cn, c2 = float(cam @ n), float(cam @ cam)

    def roots(R):
        disc = cn * cn - (c2 - R * R)
        if disc <= 0:
            return None
        q = math.sqrt(disc)
        return -cn - q, -cn + q

    outer = roots(r_out)
    if outer is None:
        return []
    inner = roots(r_in)
    a, b = max(outer[0], 0.0), outer[1]
    if inner is None or inner[1] <= a:
        return [(a, b)] if b > a else []
    return [(a, max(a, inner[0])), (min(b, inner[1]), b)]


def ray_dirs(oracle, d):
    """Camera position and unit direction of every ray (straight lines in flat space)."""
    st, _ = oracle.trace(d, {}, precision=1)
    cam = np.array([d.cam_pos[0], d.cam_pos[1], d.cam_pos[2]], dtype=np.float64)
    end = st[:, 3:6]
    n = end - cam
    return cam, n / np.linalg.norm(n, axis=1, keepdims=True)


def test_flat_uniform_plasma_gives_the_chord_length(oracle):
    d = flat_frame(5, 5, fov_deg=30.0)
    scenes.set_emission(d, abi.EMISSION_DISK, index=0.0, height=1e4, r_in=3.0, r_out=6.0)
    em = oracle.trace_emission(d, {}, precision=1)
    cam, n = ray_dirs(oracle, d)
    assert np.allclose(em[:, 2], 1.0)  # static camera in flat space measures the traced frequency 1
    for k in range(d.nrays):
        L = sum(b - a for a, b in shell_segments(cam, n[k], 3.0, 6.0))
        assert abs(em[k, 0] - L) <= 0.03, (k, em[k, 0], L)
    assert em[:, 0].max() > 5.0  # some rays do cross the shell


def test_flat_grey_absorption(oracle):
    kappa = 0.3
    d = flat_frame(3, 3, fov_deg=8.0, hmax=0.002)  # boundary error of the step sum: ~kappa * h per shell crossing
    scenes.set_emission(d, abi.EMISSION_DISK, index=0.0, height=1e4, r_in=0.5, r_out=5.0, absorb=kappa)
    em = oracle.trace_emission(d, {}, precision=1)
    cam, n = ray_dirs(oracle, d)
    for k in range(d.nrays):
        segs = shell_segments(cam, n[k], 0.5, 5.0)
        I, tau = 0.0, 0.0
        for a, b in segs:
            I += math.exp(-tau) * (1.0 - math.exp(-kappa * (b - a))) / kappa
            tau += kappa * (b - a)
        assert em[k, 1] == pytest.approx(math.exp(-tau), rel=1e-3), k
        assert em[k, 0] == pytest.approx(I, rel=2e-3), k


@pytest.mark.parametrize("beta,alpha", [(0.5, 0.0), (-0.5, 0.0), (0.3, 1.0)])
def test_flat_doppler_factor(oracle, beta, alpha):
    kappa = 0.05
    nodes = np.ones((3, 3, 3), dtype=np.float32)
    vel = np.zeros((3, 3, 3, 3), dtype=np.float32)
    vel[..., 0] = beta
    oracle.set_plasma(nodes, (-20, -20, -20), (20, 20, 20), velocity=vel)
    try:
        d = flat_frame()
        scenes.set_emission(d, abi.EMISSION_GRID, r_in=2.0, r_out=7.0, spectral_index=alpha, absorb=kappa)
        em = oracle.trace_emission(d, {}, precision=1)
    finally:
        oracle.set_plasma(None)
    cam, n = ray_dirs(oracle, d)
    gamma = 1.0 / math.sqrt(1.0 - beta * beta)
    g = 1.0 / (gamma * (1.0 - beta * float(n[0, 0])))
    L1 = 5.0  # two segments of length 5 along the axis
    tau1 = kappa * L1 / g
    I = g ** (2 + alpha) * (1 - math.exp(-tau1)) / (kappa / g) * (1 + math.exp(-tau1))
    assert em[0, 1] == pytest.approx(math.exp(-2 * tau1), rel=2e-3)
    assert em[0, 0] == pytest.approx(I, rel=5e-3)


def test_linear_grid_is_interpolated_exactly(oracle):
    nx, ny, nz = 7, 5, 4
    lo, hi = np.array([-12.0, -11.0, -10.0]), np.array([12.0, 13.0, 10.0])
    xs = [np.linspace(lo[k], hi[k], m) for k, m in enumerate((nx, ny, nz))]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    c0, c = 2.0, np.array([0.05, -0.03, 0.02])
    dens = (c0 + c[0] * X + c[1] * Y + c[2] * Z).astype(np.float32)
    theta = np.full(dens.shape, 2.0, dtype=np.float32)
    oracle.set_plasma(dens, lo, hi, temperature=theta, velocity=np.zeros(dens.shape + (3,), np.float32))
    try:
        d = flat_frame(4, 3, fov_deg=25.0)
        scenes.set_emission(d, abi.EMISSION_GRID, r_in=1.5, r_out=9.0, temp_power=1.5)
        em = oracle.trace_emission(d, {}, precision=1)
    finally:
        oracle.set_plasma(None)
    cam, n = ray_dirs(oracle, d)
    for k in range(d.nrays):
        I = 0.0
        for a, b in shell_segments(cam, n[k], 1.5, 9.0):
            I += c0 * (b - a) + float(c @ (cam * (b - a) + n[k] * (b * b - a * a) / 2))
        assert em[k, 0] == pytest.approx(I * 2.0 ** 1.5, rel=4e-3, abs=0.02), k


def test_schwarzschild_radial_redshift(oracle):
    M, rc, r1, r2 = 1.0, 30.0, 4.0, 8.0
    oracle.set_plasma(np.ones((3, 3, 3), np.float32), (-12, -12, -12), (12, 12, 12),
                      velocity=np.zeros((3, 3, 3, 3), np.float32))
    try:
        d = scenes.make_frame(1, 1, r=rc, incl_deg=90.0, fov_deg=10.0, metric=abi.METRIC_SCHWARZSCHILD, mass=M,
                              precision=abi.PREC_FP64, background=False, hmax=0.002, tol=1e-10, max_steps=500000)
        scenes.set_emission(d, abi.EMISSION_GRID, r_in=r1, r_out=r2)
        em = oracle.trace_emission(d, {}, precision=1)
        st, _ = oracle.trace(d, {}, precision=1)
    finally:
        oracle.set_plasma(None)
    assert st[0, 2] == abi.RESULT_SUCCESS  # captured at the horizon
    I = (r2 - r1 - 2 * M * math.log(r2 / r1)) / (1 - 2 * M / rc) ** 1.5
    assert em[0, 0] == pytest.approx(I, rel=3e-3)
    assert em[0, 2] == pytest.approx(1.0 / math.sqrt(1 - 2 * M / rc), rel=1e-6)  # u^t of the null ray, per static observer


def test_edge_on_disk_mirrors_with_the_flow(oracle):
    imgs = []
    for sense in (1, -1):
        d = scenes.make_frame(24, 8, r=30.0, incl_deg=90.0, fov_deg=30.0, metric=abi.METRIC_SCHWARZSCHILD,
                              precision=abi.PREC_FP64, background=False)
        scenes.set_emission(d, abi.EMISSION_DISK, index=2.0, height=0.2, r_in=3.0, r_out=12.0, sense=sense)
        imgs.append(oracle.trace_emission(d, {}, precision=1)[:, 0].reshape(8, 24))
    a, b = imgs
    assert np.allclose(a, b[:, ::-1], rtol=1e-4, atol=1e-9)
    assert not np.allclose(a, a[:, ::-1], rtol=0.05)  # beaming: one side brighter
    assert a.max() > 0


def test_emission_colour_composite(oracle):
    """GREY map: rgb = trans * colour + clamp(gain * I); a black sky leaves clamp(gain * I)."""
    d = flat_frame(3, 3, fov_deg=20.0)
    scenes.set_emission(d, abi.EMISSION_DISK, index=0.0, height=1e4, r_in=2.0, r_out=6.0, gain=0.1,
                        colormap=abi.CMAP_GREY, absorb=0.1)
    em = oracle.trace_emission(d, {}, precision=1)
    _, rgb = oracle.trace(d, {}, precision=1)
    want = np.clip(0.1 * em[:, 0], 0, 1)
    assert np.allclose(rgb, want[:, None], atol=1e-6)
    d.emis.colormap = abi.CMAP_AFMHOT
    _, rgb = oracle.trace(d, {}, precision=1)
    x = 0.1 * em[:, 0]
    assert np.allclose(rgb, np.clip(np.stack([2 * x, 2 * x - 0.5, 2 * x - 1], 1), 0, 1), atol=1e-6)
