"""prr-b200: B200-native ParRelRay hot path (geodesic ray tracing through
flat / Schwarzschild / Kerr spacetimes, textured spheres, SSAA and FXAA).

The product is the C ABI of include/prr.h, implemented by
_lib/libprr_b200.so (CUDA for sm_100a).  This package is a thin Python view
of that ABI (numpy in, numpy out) plus the workload builders in scenes.py.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .abi import FrameDesc, LaunchConfig, PrrError, Stats

__all__ = ["Context", "Deck", "FrameDesc", "Graph", "LaunchConfig", "PrrError", "Stats", "abi", "load_image",
           "write_png"]


def _frames_array(frames) -> tuple[C.Array, list[FrameDesc]]:
    if isinstance(frames, FrameDesc):
        frames = [frames]
    frames = list(frames)
    arr = (FrameDesc * len(frames))(*frames)
    return arr, frames


class Context:
    """One device context (prr_create/prr_destroy)."""

    def __init__(self, device: int = 0):
        self.lib = abi.load()
        h = C.c_void_p()
        st = self.lib.prr_create(device, C.byref(h))
        if st != abi.OK:
            raise PrrError(st, self.lib.prr_status_string(st).decode())
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.prr_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        abi.check(st, self.h)

    def upload_texture(self, tex_id: int, rgba8: np.ndarray) -> None:
        a = np.ascontiguousarray(rgba8, dtype=np.uint8)
        if a.ndim != 3 or a.shape[2] != 4:
            raise ValueError("texture must be an (h, w, 4) uint8 array")
        self._check(self.lib.prr_upload_texture(self.h, tex_id, a.ctypes.data_as(abi._u8p), a.shape[1], a.shape[0]))

    def upload_textures(self, textures: dict[int, np.ndarray]) -> None:
        for k, v in textures.items():
            self.upload_texture(k, v)

    def upload_plasma(self, density: np.ndarray, lo, hi, temperature: np.ndarray | None = None,
                      velocity: np.ndarray | None = None) -> None:
        """The plasma grid of GRID emission (prr_upload_plasma): density and temperature as (nz, ny, nx)
        arrays, velocity as (nz, ny, nx, 3) (coordinate velocity dx/dt), on nodes spanning the box lo..hi."""
        n = np.ascontiguousarray(density, dtype=np.float32)
        if n.ndim != 3:
            raise ValueError("density must be an (nz, ny, nx) array")
        t = None if temperature is None else np.ascontiguousarray(temperature, dtype=np.float32)
        v = None if velocity is None else np.ascontiguousarray(velocity, dtype=np.float32)
        if t is not None and t.shape != n.shape:
            raise ValueError("temperature must have the density's shape")
        if v is not None and v.shape != n.shape + (3,):
            raise ValueError("velocity must be an (nz, ny, nx, 3) array")
        d = abi.PlasmaDesc()
        d.nz, d.ny, d.nx = n.shape
        d.lo[:] = [float(x) for x in lo]
        d.hi[:] = [float(x) for x in hi]
        d.density = n.ctypes.data_as(abi._fp)
        d.temperature = t.ctypes.data_as(abi._fp) if t is not None else None
        d.velocity = v.ctypes.data_as(abi._fp) if v is not None else None
        self._check(self.lib.prr_upload_plasma(self.h, C.byref(d)))

    def set_schedule(self, schedule: int, cfg: LaunchConfig | None = None) -> None:
        self._check(self.lib.prr_set_schedule(self.h, schedule, C.byref(cfg) if cfg else None))

    def launch_config(self) -> LaunchConfig:
        cfg = LaunchConfig()
        self._check(self.lib.prr_get_launch_config(self.h, C.byref(cfg)))
        return cfg

    def set_option(self, option: int, value: int) -> None:
        self._check(self.lib.prr_set_option(self.h, option, value))

    def autotune(self, frame: FrameDesc) -> LaunchConfig:
        cfg = LaunchConfig()
        self._check(self.lib.prr_autotune(self.h, C.byref(frame), C.byref(cfg)))
        return cfg

    def measure_peak(self) -> tuple[float, float]:
        f32, f64 = C.c_double(), C.c_double()
        self._check(self.lib.prr_measure_peak(self.h, C.byref(f32), C.byref(f64)))
        return f32.value, f64.value

    def check_recip(self, x: np.ndarray) -> np.ndarray:
        """prr_check_recip: (n, 4) float64 of the device's FP64 1/x, 1/sqrt(x) and FP32 1/x,
        1/sqrt(x) as the PHYSICAL kernels compute them."""
        xs = np.ascontiguousarray(x, dtype=np.float64).ravel()
        out = np.empty((xs.size, 4), dtype=np.float64)
        self._check(self.lib.prr_check_recip(self.h, xs.ctypes.data_as(abi._dp), xs.size, out.ctypes.data_as(abi._dp)))
        return out

    def render(self, frames, want_float: bool = False, out8: np.ndarray | None = None):
        """Renders one or more frames; returns (list of uint8 (h, w, 3)
        images, list of float32 images or None, Stats).  `out8` may supply
        the flat uint8 output buffer (e.g. pinned host memory)."""
        arr, fl = _frames_array(frames)
        npx = sum(max(f.width, 0) * max(f.height, 0) for f in fl)  # the library validates sizes
        if out8 is None:
            out8 = np.empty(npx * 3, dtype=np.uint8)
        elif out8.dtype != np.uint8 or out8.size < npx * 3 or not out8.flags.c_contiguous:
            raise ValueError("out8 must be a contiguous uint8 array of at least 3*pixels elements")
        outf = np.empty(npx * 3, dtype=np.float32) if want_float else None
        stats = Stats()
        self._check(self.lib.prr_render(self.h, arr, len(fl), out8.ctypes.data_as(abi._u8p),
                                        outf.ctypes.data_as(abi._fp) if want_float else None, C.byref(stats)))
        imgs8, imgsf, off = [], [], 0
        for f in fl:
            n = f.width * f.height * 3
            imgs8.append(out8[off:off + n].reshape(f.height, f.width, 3))
            if want_float:
                imgsf.append(outf[off:off + n].reshape(f.height, f.width, 3))
            off += n
        return imgs8, (imgsf if want_float else None), stats

    def render_device(self, frames, d_rgb8: int, d_rgbf: int | None = None, stream: int | None = None) -> None:
        """Asynchronous render into device buffers (raw CUDA pointers)."""
        arr, fl = _frames_array(frames)
        self._check(self.lib.prr_render_device(self.h, arr, len(fl), C.c_void_p(d_rgb8),
                                               C.c_void_p(d_rgbf) if d_rgbf else None,
                                               C.c_void_p(stream) if stream else None))

    def load_metric_plugin(self, path) -> int:
        """prr_load_metric_plugin: returns the metric id for frames."""
        mid = C.c_int()
        self._check(self.lib.prr_load_metric_plugin(self.h, str(path).encode(), C.byref(mid)))
        return mid.value

    def run_deck(self, path, first: int = 0, count: int = -1, prefix: str | None = None, batch: int = 16) -> Stats:
        """prr_run_deck: renders a deck's frames to <prefix>image_<i>.png."""
        st = Stats()
        self._check(self.lib.prr_run_deck(self.h, str(path).encode(), first, count,
                                          prefix.encode() if prefix is not None else None, batch, C.byref(st)))
        return st

    def trace_rays(self, frame: FrameDesc):
        """Per-ray final states (n, 12) float32 and per-sample colours (n, 3)."""
        n = frame.nrays
        state = np.empty((n, 12), dtype=np.float32)
        rgb = np.empty((n, 3), dtype=np.float32)
        stats = Stats()
        self._check(self.lib.prr_trace_rays(self.h, C.byref(frame), state.ctypes.data_as(abi._fp),
                                            rgb.ctypes.data_as(abi._fp), C.byref(stats)))
        return state, rgb, stats

    def trace_rays_f64(self, frame: FrameDesc):
        n = frame.nrays
        state = np.empty((n, 12), dtype=np.float64)
        rgb = np.empty((n, 3), dtype=np.float64)
        stats = Stats()
        self._check(self.lib.prr_trace_rays_f64(self.h, C.byref(frame), state.ctypes.data_as(abi._dp),
                                                rgb.ctypes.data_as(abi._dp), C.byref(stats)))
        return state, rgb, stats

    def adjoint(self, frame: FrameDesc, dl_dimage: np.ndarray, sphere_index: int = -1):
        """prr_adjoint: d(loss)/d(spin, mass, inclination, camera r, sphere
        phase) for dl_dimage = d(loss)/d(float image), shape (h, w, 3).
        Returns (float64 array of 5, Stats)."""
        dl = np.ascontiguousarray(dl_dimage, dtype=np.float32)
        if dl.size != frame.width * frame.height * 3:
            raise ValueError("dl_dimage must hold width*height*3 values")
        grads = np.zeros(5, dtype=np.float64)
        stats = Stats()
        self._check(self.lib.prr_adjoint(self.h, C.byref(frame), dl.ctypes.data_as(abi._fp), int(sphere_index),
                                         grads.ctypes.data_as(abi._dp), C.byref(stats)))
        return grads, stats


class Graph:
    """A batch of frames recorded into a CUDA graph (prr_graph_*): device
    outputs given as raw pointers; replay with launch(stream)."""

    def __init__(self, ctx: Context, frames, d_rgb8: int | None, d_rgbf: int | None = None):
        self.ctx = ctx
        self.lib = ctx.lib
        arr, fl = _frames_array(frames)
        self.nframes = len(fl)
        h = C.c_void_p()
        ctx._check(self.lib.prr_graph_create(ctx.h, arr, len(fl), C.c_void_p(d_rgb8) if d_rgb8 else None,
                                             C.c_void_p(d_rgbf) if d_rgbf else None, C.byref(h)))
        self.h = h

    def set_frames(self, frames) -> None:
        arr, fl = _frames_array(frames)
        self.ctx._check(self.lib.prr_graph_set_frames(self.h, arr, len(fl)))

    def launch(self, stream: int | None = None) -> None:
        self.ctx._check(self.lib.prr_graph_launch(self.h, C.c_void_p(stream) if stream else None))

    def stats(self) -> Stats:
        st = Stats()
        self.ctx._check(self.lib.prr_graph_stats(self.h, C.byref(st)))
        return st

    def launch_config(self) -> LaunchConfig:
        cfg = LaunchConfig()
        self.ctx._check(self.lib.prr_graph_get_launch_config(self.h, C.byref(cfg)))
        return cfg

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.prr_graph_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Deck:
    """A reference-format deck (prr_deck_*): getters with the reference's
    semantics and the frame descriptors it defines."""

    def __init__(self, path=None, text: str | None = None):
        self.lib = abi.load()
        h = C.c_void_p()
        if text is not None:
            st = self.lib.prr_deck_parse_string(text.encode(), C.byref(h))
            if st != abi.OK:
                raise PrrError(st, "deck text could not be parsed")
        else:
            err = C.create_string_buffer(512)
            st = self.lib.prr_deck_load(str(path).encode(), C.byref(h), err, 512)
            if st != abi.OK:
                raise PrrError(st, err.value.decode())
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.prr_deck_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def has_block(self, block: str) -> bool:
        return bool(self.lib.prr_deck_has_block(self.h, block.encode()))

    def has(self, block: str, key: str) -> bool:
        return bool(self.lib.prr_deck_has(self.h, block.encode(), key.encode()))

    def get(self, block: str, key: str) -> str:
        n = self.lib.prr_deck_get(self.h, block.encode(), key.encode(), None, 0)
        buf = C.create_string_buffer(n + 1)
        self.lib.prr_deck_get(self.h, block.encode(), key.encode(), buf, n + 1)
        return buf.raw[:n].decode("utf-8", "surrogateescape")

    def geti(self, block: str, key: str) -> int:
        return self.lib.prr_deck_geti(self.h, block.encode(), key.encode())

    def getf(self, block: str, key: str, default: float = 0.0) -> float:
        return self.lib.prr_deck_getf(self.h, block.encode(), key.encode(), default)

    @property
    def frame_count(self) -> int:
        return self.lib.prr_deck_frame_count(self.h)

    @property
    def sphere_count(self) -> int:
        return self.lib.prr_deck_sphere_count(self.h)

    def frame(self, i: int) -> FrameDesc:
        d = FrameDesc()
        err = C.create_string_buffer(512)
        st = self.lib.prr_deck_frame(self.h, i, C.byref(d), err, 512)
        if st != abi.OK:
            raise PrrError(st, err.value.decode())
        return d


def load_image(path) -> np.ndarray:
    """prr_image_load: (h, w, 4) uint8 RGBA."""
    lib = abi.load()
    p, w, h = abi._u8p(), C.c_int(), C.c_int()
    err = C.create_string_buffer(512)
    st = lib.prr_image_load(str(path).encode(), C.byref(p), C.byref(w), C.byref(h), err, 512)
    if st != abi.OK:
        raise PrrError(st, err.value.decode())
    try:
        return np.ctypeslib.as_array(p, shape=(h.value, w.value, 4)).copy()
    finally:
        lib.prr_image_free(p)


def write_png(path, rgb8: np.ndarray) -> None:
    a = np.ascontiguousarray(rgb8, dtype=np.uint8)
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError("need an (h, w, 3) uint8 array")
    abi.check(abi.load().prr_png_write(str(path).encode(), a.ctypes.data_as(abi._u8p), a.shape[1], a.shape[0]))
