"""Test-side access to the CPU oracles (test infrastructure only).

* `Oracle`  - the CPU restatement, oracle/_build/libprr_oracle.so
              (oracle/prr_oracle.cpp), REFERENCE and PHYSICAL modes.
* `RefHost` - the reference's own sources built for the host,
              oracle/_ref/libprr_ref_{schw,flat,kerr}.so (oracle/ref/), driven
              through a reference-format deck written by `write_deck`.
"""
from __future__ import annotations

import ctypes as C
import os
import random
import string
from pathlib import Path

import numpy as np

from parrelray_b200 import abi

REPO = Path(__file__).resolve().parents[1]
ORACLE_LIB = REPO / "oracle" / "_build" / "libprr_oracle.so"
REF_DIR = REPO / "oracle" / "_ref"

_u8pp = C.POINTER(C.POINTER(C.c_uint8))
_ip = C.POINTER(C.c_int)


def ref_available(metric_tag: str = "schw") -> bool:
    return (REF_DIR / f"libprr_ref_{metric_tag}.so").exists()


class TexTable:
    """PRR_MAX_TEXTURES-long pointer/size arrays for the oracle ABI."""

    def __init__(self, textures: dict[int, np.ndarray]):
        self.keep = {k: np.ascontiguousarray(v, dtype=np.uint8) for k, v in textures.items()}
        self.ptrs = (C.POINTER(C.c_uint8) * abi.PRR_MAX_TEXTURES)()
        self.w = (C.c_int * abi.PRR_MAX_TEXTURES)()
        self.h = (C.c_int * abi.PRR_MAX_TEXTURES)()
        for k, v in self.keep.items():
            self.ptrs[k] = v.ctypes.data_as(C.POINTER(C.c_uint8))
            self.h[k], self.w[k] = v.shape[0], v.shape[1]


class Oracle:
    def __init__(self, path: Path = ORACLE_LIB):
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `python -m parrelray_b200.build --oracle`")
        lib = C.CDLL(str(path))
        lib.prr_oracle_trace.restype = C.c_int
        lib.prr_oracle_trace.argtypes = [C.POINTER(abi.FrameDesc), _u8pp, _ip, _ip, C.c_int,
                                         C.POINTER(C.c_longlong), C.c_longlong, C.c_int,
                                         C.POINTER(C.c_double), C.POINTER(C.c_float)]
        lib.prr_oracle_post.restype = C.c_int
        lib.prr_oracle_post.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]
        lib.prr_oracle_geod.restype = None
        lib.prr_oracle_geod.argtypes = [C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double)]
        lib.prr_oracle_grad.restype = C.c_int
        lib.prr_oracle_grad.argtypes = [C.POINTER(abi.FrameDesc), _u8pp, _ip, _ip, C.POINTER(C.c_float), C.c_int,
                                        C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
        lib.prr_oracle_metric.restype = None
        lib.prr_oracle_metric.argtypes = [C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.prr_oracle_trace_emission.restype = C.c_int
        lib.prr_oracle_trace_emission.argtypes = [C.POINTER(abi.FrameDesc), _u8pp, _ip, _ip, C.c_int,
                                                  C.POINTER(C.c_longlong), C.c_longlong, C.c_int, C.POINTER(C.c_double)]
        lib.prr_oracle_set_plasma.restype = C.c_int
        lib.prr_oracle_set_plasma.argtypes = [C.POINTER(abi.PlasmaDesc)]
        lib.prr_oracle_make_texture.restype = C.c_int
        lib.prr_oracle_make_texture.argtypes = [C.c_int, C.c_uint32, C.c_int, C.c_int, C.POINTER(C.c_uint8)]
        self.lib = lib
        self._plasma_keep = None

    def make_texture(self, kind: int, seed: int, w: int, h: int) -> np.ndarray:
        """The seeded procedural texture of prr_make_texture, made without the product library."""
        out = np.empty((h, w, 4), dtype=np.uint8)
        if self.lib.prr_oracle_make_texture(kind, seed, w, h, out.ctypes.data_as(C.POINTER(C.c_uint8))):
            raise ValueError("bad texture request")
        return out

    def standard_textures(self) -> dict[int, np.ndarray]:
        """scenes.standard_textures() (the starfield and the three sphere textures), made here."""
        from parrelray_b200 import scenes

        tex = {scenes.SKY_ID: self.make_texture(1, 1234, *scenes.SKY_TEX_SIZE)}
        for k in range(3):
            tex[scenes.SPHERE_ID0 + k] = self.make_texture(0, 100 + k, *scenes.SPHERE_TEX_SIZE)
        return tex

    def set_plasma(self, density=None, lo=None, hi=None, temperature=None, velocity=None) -> None:
        """The plasma grid of GRID emission, as Context.upload_plasma takes it; no density clears it."""
        if density is None:
            self.lib.prr_oracle_set_plasma(None)
            self._plasma_keep = None
            return
        n = np.ascontiguousarray(density, dtype=np.float32)
        t = None if temperature is None else np.ascontiguousarray(temperature, dtype=np.float32)
        v = None if velocity is None else np.ascontiguousarray(velocity, dtype=np.float32)
        d = abi.PlasmaDesc()
        d.nz, d.ny, d.nx = n.shape
        d.lo[:] = [float(x) for x in lo]
        d.hi[:] = [float(x) for x in hi]
        fp = C.POINTER(C.c_float)
        d.density = n.ctypes.data_as(fp)
        d.temperature = t.ctypes.data_as(fp) if t is not None else None
        d.velocity = v.ctypes.data_as(fp) if v is not None else None
        if self.lib.prr_oracle_set_plasma(C.byref(d)):
            raise ValueError("oracle rejected the plasma grid")
        self._plasma_keep = (n, t, v)

    def trace_emission(self, d: abi.FrameDesc, textures, precision: int = 0, ids=None, nthreads: int | None = None):
        """(n, 3) float64 per ray: emission intensity I, transmittance, camera frequency nu_cam."""
        tt = TexTable(textures)
        if ids is None:
            n, idp = d.nrays, None
        else:
            ids = np.ascontiguousarray(ids, dtype=np.int64)
            n, idp = len(ids), ids.ctypes.data_as(C.POINTER(C.c_longlong))
        out = np.zeros((n, 3), dtype=np.float64)
        rc = self.lib.prr_oracle_trace_emission(C.byref(d), tt.ptrs, tt.w, tt.h, precision, idp, n,
                                                nthreads or os.cpu_count(), out.ctypes.data_as(C.POINTER(C.c_double)))
        if rc:
            raise ValueError("oracle rejected the frame")
        return out

    def trace(self, d: abi.FrameDesc, textures: dict[int, np.ndarray], precision: int = 0, ids=None,
              nthreads: int | None = None):
        """(state (n, 13) float64, rgb (n, 3) float32) for the rays `ids`
        (default: every ray of the frame).  state columns: uv.x uv.y result
        r.x r.y r.z r.w u.x u.y u.z u.w accepted attempts."""
        tt = TexTable(textures)
        if ids is None:
            n = d.nrays
            idp = None
        else:
            ids = np.ascontiguousarray(ids, dtype=np.int64)
            n = len(ids)
            idp = ids.ctypes.data_as(C.POINTER(C.c_longlong))
        state = np.zeros((n, 13), dtype=np.float64)
        rgb = np.zeros((n, 3), dtype=np.float32)
        rc = self.lib.prr_oracle_trace(C.byref(d), tt.ptrs, tt.w, tt.h, precision, idp, n, nthreads or os.cpu_count(),
                                       state.ctypes.data_as(C.POINTER(C.c_double)), rgb.ctypes.data_as(C.POINTER(C.c_float)))
        if rc:
            raise ValueError("oracle rejected the frame")
        return state, rgb

    def post(self, rgb: np.ndarray, w: int, h: int, samples: int, fxaa: bool) -> np.ndarray:
        rgb = np.ascontiguousarray(rgb, dtype=np.float32)
        out = np.zeros((h, w, 3), dtype=np.float32)
        self.lib.prr_oracle_post(rgb.ctypes.data_as(C.POINTER(C.c_float)), w, h, samples, 1 if fxaa else 0,
                                 out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def render(self, d: abi.FrameDesc, textures, precision: int = 0):
        state, rgb = self.trace(d, textures, precision)
        img = self.post(rgb, d.width, d.height, d.samples, bool(d.fxaa))
        return state, rgb, img

    def grad(self, d: abi.FrameDesc, textures, dL_dimage: np.ndarray, sphere_index: int = 0, params=None,
             nthreads: int | None = None):
        """FP64 forward-mode gradient (spin, mass, inclination, camera r,
        sphere phase) of sum(dL_dimage * image); returns (grads, image)."""
        tt = TexTable(textures)
        g = np.zeros(5, dtype=np.float64)
        img = np.zeros((d.height, d.width, 3), dtype=np.float64)
        dl = np.ascontiguousarray(dL_dimage, dtype=np.float32)
        pp = (C.c_double * 5)(*params) if params is not None else None
        loss = C.c_double()
        sig = np.zeros((d.height, d.width), dtype=np.int64)
        rc = self.lib.prr_oracle_grad(C.byref(d), tt.ptrs, tt.w, tt.h, dl.ctypes.data_as(C.POINTER(C.c_float)),
                                      sphere_index, nthreads or os.cpu_count(), g.ctypes.data_as(C.POINTER(C.c_double)),
                                      img.ctypes.data_as(C.POINTER(C.c_double)), pp, C.byref(loss),
                                      sig.ctypes.data_as(C.POINTER(C.c_longlong)))
        if rc:
            raise ValueError("oracle rejected the frame for gradients")
        self.last_loss, self.last_sig = loss.value, sig
        return g, img

    def geod(self, metric: int, M: float, a: float, p, u, refmode: bool = False) -> np.ndarray:
        pa = (C.c_double * 4)(*p)
        ua = (C.c_double * 4)(*u)
        out = (C.c_double * 4)()
        self.lib.prr_oracle_geod(metric, M, a, pa, ua, 1 if refmode else 0, out)
        return np.array(out[:])

    def metric(self, metric: int, M: float, a: float, p) -> np.ndarray:
        pa = (C.c_double * 4)(*p)
        g = (C.c_double * 16)()
        self.lib.prr_oracle_metric(metric, M, a, pa, g)
        return np.array(g[:]).reshape(4, 4)


def kerr_criticality(state: np.ndarray, M: float, a: float, n_grid: int = 48) -> np.ndarray:
    """Per ray, |min over r in [r_+, 6M] of R(r)/r^4|, with R the Boyer-Lindquist radial potential
    (r^2 + a^2 - a xi)^2 - Delta (eta + (xi - a)^2) of the ray's conserved xi = L_z/E and
    eta = Q/E^2 (Carter), evaluated from a Kerr-Schild state (columns 3..10 of Oracle.trace /
    Context.trace_rays: x y z t, u^x u^y u^z u^t).  A photon orbit is a double root of R; for
    Schwarzschild min R/r^4 = 1 - (b/b_c)^2, so a value below 2 delta marks a ray within a
    relative delta of the critical impact parameter.  The same test as the renderer's
    near_critical (parrelray_b200/csrc/phys_stepper.cuh), vectorised in FP64."""
    st = np.asarray(state, dtype=np.float64)
    x, y, z = st[:, 3], st[:, 4], st[:, 5]
    u = st[:, 7:11]
    R2 = x * x + y * y + z * z
    bq = R2 - a * a
    r = np.sqrt(0.5 * (bq + np.sqrt(bq * bq + 4 * a * a * z * z)))
    q = r * r + a * a
    f = 2 * M * r ** 3 / (r ** 4 + a * a * z * z)
    l = np.stack([(r * x + a * y) / q, (r * y - a * x) / q, z / r, np.ones_like(r)], 1)
    eta = np.array([1.0, 1.0, 1.0, -1.0])
    L = np.sum(l * u, 1)
    p = eta * u + (f * L)[:, None] * l  # p_m = g_mn u^n
    E = -p[:, 3]
    Lz = x * p[:, 1] - y * p[:, 0]
    ct = z / r
    st2 = np.maximum(1.0 - ct * ct, 1e-300)
    sn = np.sqrt(st2)
    pth = (ct / sn) * (x * p[:, 0] + y * p[:, 1]) - r * sn * p[:, 2]
    Q = pth * pth + ct * ct * (-a * a * E * E + Lz * Lz / st2)
    xi, et = Lz / E, Q / (E * E)
    rp = M + np.sqrt(max(M * M - a * a, 0.0))
    rr = np.linspace(rp * 1.0001, 6.0 * M, n_grid + 1)[None, :]
    A = rr * rr + a * a - a * xi[:, None]
    D = rr * rr - 2 * M * rr + a * a
    pot = (A * A - D * (et[:, None] + (xi[:, None] - a) ** 2)) / rr ** 4
    return np.abs(pot.min(axis=1))


def _safe_dir(base: Path) -> Path:
    """The reference's deck parser treats any line with '_' as a block header
    (main/io.h:33), so paths written into a deck must not contain '_'."""
    base.mkdir(parents=True, exist_ok=True)
    name = "prr" + "".join(random.choice(string.ascii_lowercase + string.digits) for _ in range(10))
    d = base / name
    d.mkdir()
    assert "_" not in str(d) and "<" not in str(d) and ">" not in str(d), d
    return d


def write_ppm(path: Path, rgba: np.ndarray) -> None:
    h, w = rgba.shape[:2]
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(np.ascontiguousarray(rgba[:, :, :3]).tobytes())


def g9(x: float) -> str:
    return "%.9g" % float(np.float32(x))


def write_deck(base: Path, d: abi.FrameDesc, textures: dict[int, np.ndarray], *, fov_deg: float, a_deg: float,
               b_deg: float, solver: str = "rkf") -> Path:
    """Writes sim/traj/scene decks reproducing `d` for the reference.  The
    camera angles and FOV are passed in degrees (the deck's unit); `d` must
    have been built from the same degrees."""
    root = _safe_dir(base)
    tex_paths = {}
    for k, v in textures.items():
        p = root / f"tex{k}.ppm"
        write_ppm(p, v)
        tex_paths[k] = p
    sim = root / "sim.params"
    traj = root / "traj.params"
    scene = root / "scene.params"
    bimage = str(tex_paths[d.background_id]) if d.background_id >= 0 else ""
    ssaa = "none" if d.ssaa == abi.SSAA_NONE else "regular"
    sim.write_text("\n".join([
        "_tracer_",
        f"<solver> = <{solver}>",
        f"<hmin> = <{g9(d.hmin)}>",
        f"<h> = <{g9(d.h)}>",
        f"<hmax> = <{g9(d.hmax)}>",
        f"<eps> = <{g9(d.eps)}>",
        f"<rout1> = <{g9(d.rout)}>",
        f"<rout2> = <{g9(d.rout)}>",
        f"<bimage1> = <{bimage}>",
        "<bimage2> = <>",
        f"<out> = <{root}/>",
        f"<traj> = <{traj}>",
        f"<scene> = <{scene}>",
        "",
        "_spacetime_",
        "<hasBlackHole> = <1>",
        f"<mass> = <{g9(d.mass)}>",
        f"<spin> = <{g9(d.spin)}>",
        "<charge> = <0>",
        "",
        "_camera_",
        f"<vfov> = <{g9(fov_deg)}>",
        f"<width> = <{d.width}>",
        f"<height> = <{d.height}>",
        f"<SSAA> = <{ssaa}>",
        f"<SSAAsamples> = <{d.samples}>",
        "",
    ]))
    traj.write_text("\n".join([
        "_frame0_",
        f"<x> = <{g9(d.cam_pos[0])}>",
        f"<y> = <{g9(d.cam_pos[1])}>",
        f"<z> = <{g9(d.cam_pos[2])}>",
        f"<a> = <{g9(a_deg)}>",
        f"<b> = <{g9(b_deg)}>",
        "",
    ]))
    lines = []
    for k in range(d.nspheres):
        s = d.spheres[k]
        lines += [f"_sphere{k}_", f"<tex> = <{tex_paths[s.texture_id]}>", f"<x0> = <{g9(s.center[0])}>",
                  f"<y0> = <{g9(s.center[1])}>", f"<z0> = <{g9(s.center[2])}>", f"<r0> = <{g9(s.radius)}>", ""]
    scene.write_text("\n".join(lines) + "\n")
    return sim


class RefHost:
    """The reference frame pipeline on the host (oracle/_ref)."""

    def __init__(self, metric_tag: str = "schw"):
        p = REF_DIR / f"libprr_ref_{metric_tag}.so"
        if not p.exists():
            raise FileNotFoundError(f"{p} missing: run oracle/ref/build_ref.sh")
        lib = C.CDLL(str(p))
        lib.prr_ref_load.restype = C.c_int
        lib.prr_ref_load.argtypes = [C.c_char_p]
        lib.prr_ref_info.restype = None
        lib.prr_ref_info.argtypes = [_ip, _ip, _ip]
        fp = C.POINTER(C.c_float)
        lib.prr_ref_frame.restype = C.c_double
        lib.prr_ref_frame.argtypes = [C.c_int, C.c_int, C.c_int, fp, fp, fp, fp]
        lib.prr_ref_prepare.restype = C.c_int
        lib.prr_ref_prepare.argtypes = [C.c_int, C.c_int]
        lib.prr_ref_trace_blocks.restype = C.c_double
        lib.prr_ref_trace_blocks.argtypes = [C.c_int, C.c_int, _ip, _ip]
        lib.prr_ref_ray_result.restype = C.c_int
        lib.prr_ref_ray_result.argtypes = [C.c_longlong]
        self.lib = lib

    def prepare(self, frame: int = 0, nthreads: int | None = None) -> None:
        assert self.lib.prr_ref_prepare(frame, nthreads or os.cpu_count()) == 0

    def trace_blocks(self, bx, rows, nthreads: int | None = None) -> float:
        """Traces 8-ray blocks (see oracle/ref/ref_driver.cpp); returns seconds."""
        bx = np.ascontiguousarray(bx, dtype=np.int32)
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        return self.lib.prr_ref_trace_blocks(nthreads or os.cpu_count(), len(bx), bx.ctypes.data_as(_ip),
                                             rows.ctypes.data_as(_ip))

    def load(self, deck: Path) -> int:
        return self.lib.prr_ref_load(str(deck).encode())

    def frame(self, frame: int = 0, nthreads: int | None = None, rows_stride: int = 1, fxaa: bool = False):
        w, h, s = C.c_int(), C.c_int(), C.c_int()
        self.lib.prr_ref_info(C.byref(w), C.byref(h), C.byref(s))
        n = w.value * h.value * s.value
        state = np.zeros((n, 11), dtype=np.float32)
        rgb = np.zeros((n, 3), dtype=np.float32)
        img = np.zeros((h.value, w.value, 3), dtype=np.float32)
        fx = np.zeros((h.value, w.value, 3), dtype=np.float32) if fxaa else None
        fp = C.POINTER(C.c_float)
        secs = self.lib.prr_ref_frame(frame, nthreads or os.cpu_count(), rows_stride, state.ctypes.data_as(fp),
                                      rgb.ctypes.data_as(fp), img.ctypes.data_as(fp),
                                      fx.ctypes.data_as(fp) if fxaa else None)
        return {"state": state, "rgb": rgb, "image": img, "fxaa": fx, "seconds": secs}
