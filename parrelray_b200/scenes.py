"""Frame descriptors for the standard workloads and the deck-style camera
mapping.

Camera placement follows the reference: a camera at distance r and
inclination i (angle from +z) sits at (r sin i, 0, r cos i) and looks at the
origin with yaw a = 180 deg and pitch b = i - 90 deg (Camera::rayDir_Spherical,
main/Camera.h:39-42).  Angles given in degrees are converted exactly as
prr.cpp:195,246-247 converts deck values: float(deg) * M_PI / 180.0f in double,
stored as float.

Workloads (all synthetic; the reference ships no textures):
  schwarzschild_320   Schwarzschild M=1, r=30, i=85, FOV 60, 320x180, one
                      sphere (R=1) at orbit radius 10, tol 1e-6, stop at 2.01M
  kerr_1080p_ssaa4    Kerr a=0.95, r=25, i=80, FOV 50, 1920x1080, 2x2 SSAA,
                      FXAA, three spheres, tol 1e-6
  trajectory_240      240 frames 960x540, Kerr a=0.9, orbit radius 20 -> 8,
                      inclination 60 -> 88 deg
  uneven_64           64 requests: log-uniform resolutions 256^2..2048x1024,
                      a ~ U[0, 0.998], r ~ U[8, 40], i ~ U[10, 89], tol 1e-7
  kerr_512_adjoint    Kerr 512x512, one sphere R=1 at orbit radius 9
  eht_disk            Kerr a=0.94, r=50, i=17, FOV 27, pinhole, square frame, black
                      sky, emission from a thick co-rotating disk (density
                      ~ r^-3, Gaussian width 0.4 in cos theta, r_+ .. 20M,
                      spectral index 0, gain 2) - an image like the EHT's M87*
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

SPHERE_TEX_SIZE = (512, 256)
SKY_TEX_SIZE = (2048, 1024)
SKY_ID = 0          # texture id of the starfield
SPHERE_ID0 = 1      # first sphere texture id


def f32(x: float) -> float:
    return float(np.float32(x))


def deg_to_rad_f32(deg: float) -> float:
    """float(deg) * M_PI / 180.0f evaluated in double, stored as float."""
    return f32(np.float64(np.float32(deg)) * math.pi / np.float64(np.float32(180.0)))


def camera_pose(r: float, incl_deg: float) -> tuple[tuple[float, float, float], float, float]:
    """Position (floats) and yaw/pitch in degrees for a camera at (r, i)."""
    i = math.radians(incl_deg)
    pos = (f32(r * math.sin(i)), 0.0, f32(r * math.cos(i)))
    return pos, 180.0, incl_deg - 90.0


def make_frame(width: int, height: int, *, r: float, incl_deg: float, fov_deg: float, metric: int = abi.METRIC_KERR,
               mass: float = 1.0, spin: float = 0.0, samples: int = 1, fxaa: bool = False, tol: float = 1e-6,
               mode: int = abi.MODE_PHYSICAL, precision: int = abi.PREC_FP32, rout: float = 100.0,
               horizon_eps: float = 0.01, max_steps: int = 10000, spheres=(), background: bool = True,
               h: float = 0.01, hmin: float = 1e-4, hmax: float = 0.1, eps: float = 1e-3,
               bg_filter: int = abi.BG_RMS2X2) -> abi.FrameDesc:
    d = abi.fill_defaults(abi.FrameDesc())
    d.width, d.height = width, height
    d.samples = samples
    d.ssaa = abi.SSAA_NONE if samples == 1 else abi.SSAA_REGULAR
    d.vfov = deg_to_rad_f32(fov_deg)
    pos, a_deg, b_deg = camera_pose(r, incl_deg)
    d.cam_pos[0], d.cam_pos[1], d.cam_pos[2] = pos
    d.cam_alpha = deg_to_rad_f32(a_deg)
    d.cam_beta = deg_to_rad_f32(b_deg)
    d.metric = metric
    d.mass = mass
    d.spin = spin if metric == abi.METRIC_KERR else 0.0
    d.solver = abi.SOLVER_RKF45
    d.mode = mode
    d.precision = precision
    d.h, d.hmin, d.hmax, d.eps = h, hmin, hmax, eps
    d.rtol = d.atol = tol
    d.rout = rout
    d.horizon_eps = horizon_eps
    d.max_steps = max_steps
    d.background_id = SKY_ID if background else -1
    d.bg_filter = bg_filter
    d.fxaa = 1 if fxaa else 0
    d.nspheres = len(spheres)
    for k, (cx, cy, cz, rad, tex) in enumerate(spheres):
        s = d.spheres[k]
        s.center[0], s.center[1], s.center[2] = f32(cx), f32(cy), f32(cz)
        s.radius = rad
        s.texture_id = tex
    return d


def set_emission(d: abi.FrameDesc, kind: int = abi.EMISSION_DISK, *, index: float = 2.0, height: float = 0.4,
                 r_in: float = 2.0, r_out: float = 20.0, spectral_index: float = 0.0, absorb: float = 0.0,
                 gain: float = 1.0, sense: int = 1, temp_power: float = 0.0,
                 colormap: int = abi.CMAP_AFMHOT) -> abi.FrameDesc:
    """Fills the frame's emission block (prr_emission_desc)."""
    d.emission = kind
    e = d.emis
    e.index, e.height, e.r_in, e.r_out = index, height, r_in, r_out
    e.spectral_index, e.absorb, e.gain, e.sense = spectral_index, absorb, gain, sense
    e.temp_power, e.colormap = temp_power, colormap
    return d


def eht_disk(size: int = 1024, spin: float = 0.94, incl_deg: float = 17.0, r: float = 50.0, fov_deg: float = 27.0,
             precision: int = abi.PREC_FP32, samples: int = 1, gain: float = 2.0, index: float = 3.0,
             height: float = 0.4, **kw) -> abi.FrameDesc:
    """Emission from a thick disk around a Kerr hole, seen almost face-on."""
    d = make_frame(size, size, r=r, incl_deg=incl_deg, fov_deg=fov_deg, metric=abi.METRIC_KERR, spin=spin,
                   precision=precision, samples=samples, background=False)
    d.camera = abi.CAMERA_PINHOLE  # the spherical model compresses yaw by cos(pitch): near face-on it squashes the ring
    rp = 1.0 + math.sqrt(1.0 - spin * spin)
    return set_emission(d, abi.EMISSION_DISK, r_in=f32(rp), r_out=20.0, index=index, height=height, gain=gain, **kw)


def orbit_point(radius: float, phase_deg: float) -> tuple[float, float, float]:
    ph = math.radians(phase_deg)
    return radius * math.cos(ph), radius * math.sin(ph), 0.0


def schwarzschild_320(**kw) -> abi.FrameDesc:
    c = orbit_point(10.0, 60.0)
    args = dict(r=30.0, incl_deg=85.0, fov_deg=60.0, metric=abi.METRIC_SCHWARZSCHILD, mass=1.0,
                spheres=[(*c, 1.0, SPHERE_ID0)])
    args.update(kw)
    return make_frame(320, 180, **args)


# Three spheres drawn once from numpy.random.default_rng(2): radii U[0.5,1.5],
# orbit radii U[6,15], phases U[0,360) (values frozen here).
KERR_1080P_SPHERES = [(1.2, 14.0, 35.0), (0.8, 9.5, 300.0), (0.5, 6.5, 160.0)]


def kerr_1080p_ssaa4(width: int = 1920, height: int = 1080, **kw) -> abi.FrameDesc:
    sph = [(*orbit_point(orb, ph), rad, SPHERE_ID0 + k) for k, (rad, orb, ph) in enumerate(KERR_1080P_SPHERES)]
    args = dict(r=25.0, incl_deg=80.0, fov_deg=50.0, metric=abi.METRIC_KERR, mass=1.0, spin=0.95, samples=4,
                fxaa=True, spheres=sph)
    args.update(kw)
    return make_frame(width, height, **args)


def trajectory_240(n: int = 240, width: int = 960, height: int = 540, **kw) -> list[abi.FrameDesc]:
    frames = []
    for k in range(n):
        t = k / max(n - 1, 1)
        r = 20.0 + (8.0 - 20.0) * t
        inc = 60.0 + (88.0 - 60.0) * t
        args = dict(r=r, incl_deg=inc, fov_deg=60.0, metric=abi.METRIC_KERR, mass=1.0, spin=0.9,
                    spheres=[(*orbit_point(12.0, 90.0 + 1.5 * k), 1.0, SPHERE_ID0)])
        args.update(kw)
        frames.append(make_frame(width, height, **args))
    return frames


def uneven_64(n: int = 64, seed: int = 4, max_pixels: int | None = None, **kw) -> list[abi.FrameDesc]:
    rng = np.random.default_rng(seed)
    frames = []
    for _ in range(n):
        w = int(round(math.exp(rng.uniform(math.log(256), math.log(2048)))))
        hgt = int(round(math.exp(rng.uniform(math.log(256), math.log(1024)))))
        if max_pixels and w * hgt > max_pixels:
            s = math.sqrt(max_pixels / (w * hgt))
            w, hgt = max(8, int(w * s)), max(8, int(hgt * s))
        args = dict(r=float(rng.uniform(8.0, 40.0)), incl_deg=float(rng.uniform(10.0, 89.0)), fov_deg=60.0,
                    metric=abi.METRIC_KERR, mass=1.0, spin=float(rng.uniform(0.0, 0.998)), tol=1e-7)
        args.update(kw)
        frames.append(make_frame(w, hgt, **args))
    return frames


def kerr_512_adjoint(spin: float = 0.7, incl_deg: float = 60.0, r: float = 20.0, phase_deg: float = 30.0,
                     size: int = 512, **kw) -> abi.FrameDesc:
    args = dict(r=r, incl_deg=incl_deg, fov_deg=40.0, metric=abi.METRIC_KERR, mass=1.0, spin=spin,
                spheres=[(*orbit_point(9.0, phase_deg), 1.0, SPHERE_ID0)], bg_filter=abi.BG_BILINEAR)
    args.update(kw)
    return make_frame(size, size, **args)


def make_texture(kind: int, seed: int, w: int, h: int) -> np.ndarray:
    out = np.empty((h, w, 4), dtype=np.uint8)
    abi.check(abi.load().prr_make_texture(kind, seed, w, h, out.ctypes.data_as(abi._u8p)))
    return out


def standard_textures() -> dict[int, np.ndarray]:
    """Texture id -> RGBA8 array: the starfield (id 0) and three sphere textures."""
    tex = {SKY_ID: make_texture(1, 1234, *SKY_TEX_SIZE)}
    for k in range(3):
        tex[SPHERE_ID0 + k] = make_texture(0, 100 + k, *SPHERE_TEX_SIZE)
    return tex
