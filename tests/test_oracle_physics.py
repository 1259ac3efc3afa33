"""Known-answer tests of the CPU restatement's PHYSICAL mode (the FP64
reference for the Kerr and tolerance-1e-6 workloads, which the reference
itself cannot produce):

* the Kerr-Schild Christoffel contraction at a = 0 equals the reference's
  closed-form Schwarzschild acceleration (metrics/schwarzschild.cuh:90-119);
* the Christoffel table equals central finite differences of the metric;
* flat space: rays are straight lines;
* Schwarzschild: critical impact parameter b_c = 3 sqrt(3) M separates
  capture from escape;
* Kerr: E, L_z, Carter's Q and g(u,u) = 0 are conserved along rays.
"""
import math

import numpy as np
import pytest

from parrelray_b200 import abi, scenes


def ks_metric(p, M, a):
    x, y, z = p[:3]
    R2 = x * x + y * y + z * z
    b = R2 - a * a
    r2 = 0.5 * (b + math.sqrt(b * b + 4 * a * a * z * z))
    r = math.sqrt(r2)
    f = 2 * M * r2 * r / (r2 * r2 + a * a * z * z)
    l = np.array([(r * x + a * y) / (r2 + a * a), (r * y - a * x) / (r2 + a * a), z / r, 1.0])
    return np.diag([1.0, 1.0, 1.0, -1.0]) + f * np.outer(l, l), r


def schw_reference_formula(p, u, M):
    """metrics/schwarzschild.cuh:90-119 restated in float64."""
    rs = 2 * M
    x, y, z = p[:3]
    ux, uy, uz, ut = u
    r = math.sqrt(x * x + y * y + z * z)
    x2, y2, z2 = x * x, y * y, z * z
    cross = x * y * ux * uy + x * z * ux * uz + y * z * uy * uz
    pu = x * ux + y * uy + z * uz
    Phi = ((r * (x2 - 2 * y2 - 2 * z2) + rs * x2) * ux * ux + (r * (-2 * x2 + y2 - 2 * z2) + rs * y2) * uy * uy
           + (r * (-2 * x2 - 2 * y2 + z2) + rs * z2) * uz * uz + 2 * (3 * r + rs) * cross
           + r * r * (rs - r) * ut * ut + 2 * r * rs * ut * pu) * rs / (2 * r ** 6)
    dw = ((2 * r * (-x2 + y2 + z2) - rs * x2) * ux * ux + (2 * r * (x2 - y2 + z2) - rs * y2) * uy * uy
          + (2 * r * (x2 + y2 - z2) - rs * z2) * uz * uz - 2 * (4 * r + rs) * cross
          - r * r * rs * ut * ut - 2 * r * (r + rs) * ut * pu) * rs / (2 * r ** 5)
    return np.array([x * Phi, y * Phi, z * Phi, dw])


def random_state(rng, M, a, rmin=3.0, rmax=40.0):
    while True:
        p = rng.uniform(-rmax, rmax, 3)
        if rmin < np.linalg.norm(p) < rmax:
            break
    p = np.array([*p, 0.0])
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    g, _ = ks_metric(p, M, a)
    u = np.array([*d, 1.0])
    A = g[3, 3]
    B = 2 * g[3, :3] @ d
    Cc = d @ g[:3, :3] @ d
    u[3] = max((-B + math.sqrt(B * B - 4 * A * Cc)) / (2 * A), (-B - math.sqrt(B * B - 4 * A * Cc)) / (2 * A))
    return p, u


def test_kerr_at_zero_spin_is_the_reference_schwarzschild(oracle):
    rng = np.random.default_rng(1)
    for _ in range(50):
        p, u = random_state(rng, 1.0, 0.0)
        mine = oracle.geod(abi.METRIC_KERR, 1.0, 0.0, p, u)
        ref = schw_reference_formula(p, u, 1.0)
        assert np.allclose(mine, ref, rtol=1e-10, atol=1e-14 * np.abs(ref).max())


def test_christoffel_table_matches_finite_differences(oracle):
    rng = np.random.default_rng(2)
    M, a = 1.0, 0.9
    for _ in range(20):
        p, u = random_state(rng, M, a)
        h = 1e-5
        dg = np.zeros((4, 4, 4))
        for k in range(3):
            e = np.zeros(4)
            e[k] = h
            dg[:, :, k] = (oracle.metric(abi.METRIC_KERR, M, a, p + e) - oracle.metric(abi.METRIC_KERR, M, a, p - e)) / (2 * h)
        g = oracle.metric(abi.METRIC_KERR, M, a, p)
        gi = np.linalg.inv(g)
        G1 = 0.5 * (np.einsum("lnm->lmn", dg) + dg - np.einsum("mnl->lmn", dg))
        acc = -np.einsum("kl,lmn,m,n->k", gi, G1, u, u)
        mine = oracle.geod(abi.METRIC_KERR, M, a, p, u)
        assert np.allclose(mine, acc, rtol=1e-6, atol=1e-8 * np.abs(acc).max())


def physical_frame(metric, spin=0.0, W=24, H=16, r=30.0, inc=80.0, fov=40.0, tol=1e-9, rout=100.0, **kw):
    d = scenes.make_frame(W, H, r=r, incl_deg=inc, fov_deg=fov, metric=metric, mass=1.0, spin=spin,
                          mode=abi.MODE_PHYSICAL, precision=abi.PREC_FP64, tol=tol, rout=rout, background=False, **kw)
    return d


def test_flat_rays_are_straight(oracle):
    d = physical_frame(abi.METRIC_FLAT, tol=1e-10)
    st, _ = oracle.trace(d, {}, precision=1)
    x0 = np.array(d.cam_pos[:])
    assert (st[:, 2] == abi.RESULT_SUCCESS).all()
    u = st[:, 7:10]
    x = st[:, 3:6]
    # final position lies on the line x0 + s*u
    dx = x - x0
    cross = np.cross(dx, u / np.linalg.norm(u, axis=1, keepdims=True))
    assert np.abs(cross).max() < 1e-9
    assert np.allclose(np.linalg.norm(x, axis=1), 100.0, atol=0.2)
    assert np.allclose(np.linalg.norm(u, axis=1), 1.0, atol=1e-12)


def conserved(x, u, M, a):
    """E, L_z, Carter Q and g(u,u) from Kerr-Schild Cartesian states."""
    g, r = ks_metric(x, M, a)
    p = g @ u
    E = -p[3]
    Lz = x[0] * p[1] - x[1] * p[0]
    ct = x[2] / r
    st2 = 1 - ct * ct
    st = math.sqrt(st2)
    pth = (ct / st) * (x[0] * p[0] + x[1] * p[1]) - r * st * p[2]
    Q = pth * pth + ct * ct * (-a * a * E * E + Lz * Lz / st2)
    return np.array([E, Lz, Q]), u @ g @ u


def test_schwarzschild_critical_impact_parameter(oracle):
    M = 1.0
    d = physical_frame(abi.METRIC_SCHWARZSCHILD, W=40, H=40, r=60.0, inc=90.0, fov=24.0, tol=1e-10, rout=120.0,
                       horizon_eps=0.01, max_steps=100000)
    d.hmax = 0.2
    st, _ = oracle.trace(d, {}, precision=1)
    first = physical_frame(abi.METRIC_SCHWARZSCHILD, W=40, H=40, r=60.0, inc=90.0, fov=24.0, tol=1e-10, rout=120.0,
                           horizon_eps=0.01, max_steps=1)
    s1, _ = oracle.trace(first, {}, precision=1)
    bc = 3 * math.sqrt(3) * M
    checked = 0
    for i in range(len(st)):
        (E, Lz, Q), _ = conserved(s1[i, 3:7], s1[i, 7:11], M, 0.0)
        b = math.sqrt(Q + Lz * Lz) / E
        captured = st[i, 2] == abi.RESULT_SUCCESS and np.linalg.norm(st[i, 3:6]) < 3.0
        escaped = st[i, 2] == abi.RESULT_SUCCESS and np.linalg.norm(st[i, 3:6]) >= 120.0
        if b < bc * 0.995:
            assert captured, (b, st[i])
            checked += 1
        elif b > bc * 1.005:
            assert escaped, (b, st[i])
            checked += 1
    assert checked > 100


@pytest.mark.parametrize("spin", [0.5, 0.95])
def test_kerr_conserved_quantities(oracle, spin):
    M = 1.0
    kw = dict(W=20, H=12, r=25.0, inc=70.0, fov=50.0, tol=1e-9, horizon_eps=0.01)
    end, _ = oracle.trace(physical_frame(abi.METRIC_KERR, spin, max_steps=100000, **kw), {}, precision=1)
    one, _ = oracle.trace(physical_frame(abi.METRIC_KERR, spin, max_steps=1, **kw), {}, precision=1)
    n_checked = 0
    for i in range(len(end)):
        if end[i, 2] != abi.RESULT_SUCCESS or np.linalg.norm(end[i, 3:6]) < 50:
            continue  # conservation is checked on escaped rays (captured ones end at the horizon)
        c0, n0 = conserved(one[i, 3:7], one[i, 7:11], M, spin)
        c1, n1 = conserved(end[i, 3:7], end[i, 7:11], M, spin)
        scale = np.array([abs(c0[0]), abs(c0[0]) * 10, abs(c0[0]) ** 2 * 100])
        assert np.all(np.abs(c1 - c0) / scale < 1e-7), (c0, c1)
        assert abs(n0) < 1e-9 * c0[0] ** 2 and abs(n1) < 1e-6 * c0[0] ** 2
        n_checked += 1
    assert n_checked > 50


def test_stochastic_placements_and_camera_models(oracle, small_textures):
    """RANDOM samples fall inside their pixel, JITTERED ones inside their cell of the n x n grid,
    both change with the seed and repeat with it; the pinhole camera looks along its forward
    vector at the image centre, and the panorama and spherical models agree there."""
    W, H = 6, 4
    for ssaa, S in ((abi.SSAA_RANDOM, 5), (abi.SSAA_JITTERED, 4)):
        d = scenes.make_frame(W, H, r=30.0, incl_deg=80.0, fov_deg=50.0, metric=abi.METRIC_FLAT, mass=0.0,
                              samples=S, background=False)
        d.ssaa, d.ssaa_seed = ssaa, 99
        st, _ = oracle.trace(d, small_textures, precision=1)
        uv = st[:, :2].reshape(H, W, S, 2)
        px = uv[..., 0] * W - np.arange(W)[None, :, None]
        py = uv[..., 1] * H - np.arange(H)[:, None, None]
        assert np.all((px >= 0) & (px < 1 + 1e-6) & (py >= 0) & (py < 1 + 1e-6))
        if ssaa == abi.SSAA_JITTERED:
            n = 2
            i = np.arange(S) % n
            j = np.arange(S) // n
            assert np.all((np.floor(px * n) == i) | np.isclose(px * n, i + 1))
            assert np.all((np.floor(py * n) == j) | np.isclose(py * n, j + 1))
        again, _ = oracle.trace(d, small_textures, precision=1)
        assert np.array_equal(again[:, :2], st[:, :2])
        d.ssaa_seed = 100
        other, _ = oracle.trace(d, small_textures, precision=1)
        assert not np.array_equal(other[:, :2], st[:, :2])
    # image centre: pinhole and panorama look along forward = the spherical model's centre ray
    dirs = {}
    for cam in (abi.CAMERA_SPHERICAL, abi.CAMERA_PINHOLE, abi.CAMERA_PANORAMA):
        d = scenes.make_frame(1, 1, r=30.0, incl_deg=80.0, fov_deg=50.0, metric=abi.METRIC_FLAT, mass=0.0,
                              background=False, rout=1e4)
        d.camera = cam
        st, _ = oracle.trace(d, small_textures, precision=1)
        u = st[0, 7:10]
        dirs[cam] = u / np.linalg.norm(u)
    assert np.allclose(dirs[abi.CAMERA_PINHOLE], dirs[abi.CAMERA_SPHERICAL], atol=1e-6)
    assert np.allclose(dirs[abi.CAMERA_PANORAMA], dirs[abi.CAMERA_SPHERICAL], atol=1e-6)


def test_camera_models_share_orientation(oracle, small_textures):
    """For one (a, b) the three models map every screen position to nearby directions: no model is
    mirrored or tilted the other way (a mirror would put the corners ~0.8 rad apart at FOV 50)."""
    dirs = {}
    for cam in (abi.CAMERA_SPHERICAL, abi.CAMERA_PINHOLE, abi.CAMERA_PANORAMA):
        d = scenes.make_frame(3, 3, r=30.0, incl_deg=80.0, fov_deg=50.0, metric=abi.METRIC_FLAT, mass=0.0,
                              background=False, rout=1e4)
        d.camera = cam
        st, _ = oracle.trace(d, small_textures, precision=1)
        u = st[:, 7:10]
        dirs[cam] = u / np.linalg.norm(u, axis=1, keepdims=True)
    for cam in (abi.CAMERA_PINHOLE, abi.CAMERA_PANORAMA):
        ang = np.arccos(np.clip(np.sum(dirs[cam] * dirs[abi.CAMERA_SPHERICAL], axis=1), -1, 1))
        assert ang.max() < 0.15, (cam, ang)
