"""ctypes view of include/prr.h and the loader of libprr_b200.so.

Every struct here mirrors include/prr.h field for field; tests compare
ctypes.sizeof() with the library's prr_sizeof().  The library is loaded from
the package's _lib/ directory (built in-tree by parrelray_b200.build); a
missing library raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "_lib" / "libprr_b200.so"
HEADER = PKG.parent / "include" / "prr.h"

PRR_MAX_SPHERES = 8
PRR_MAX_TEXTURES = 32

# prr_status
OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_TIMEOUT, ERR_IO, ERR_UNSUPPORTED, ERR_NO_DEVICE = range(8)
# prr_result (main/base.h:37-43)
RESULT_SUCCESS, RESULT_MATH_ERROR, RESULT_IO_ERROR, RESULT_INFINITE_GEO, RESULT_INTERSECTION = range(5)
SOLVER_EULER, SOLVER_RKF45 = 0, 2
SSAA_NONE, SSAA_REGULAR, SSAA_RANDOM, SSAA_JITTERED = 0, 1, 2, 4
CAMERA_SPHERICAL, CAMERA_PINHOLE, CAMERA_PANORAMA = 0, 1, 2
METRIC_FLAT, METRIC_SCHWARZSCHILD, METRIC_KERR = 0, 1, 2
METRIC_PLUGIN0 = 16
MODE_REFERENCE, MODE_PHYSICAL = 0, 1
PREC_FP32, PREC_FP64, PREC_SPLIT = 0, 1, 2
SCHED_PLAIN, SCHED_PERSISTENT = 0, 1
BG_RMS2X2, BG_BILINEAR = 0, 1
OPT_GEOD_TABLE, OPT_WATCHDOG_CYCLES, OPT_HAMILTONIAN = 1, 2, 3
HAM_FP32, HAM_FP64 = 1, 2  # PRR_OPT_HAMILTONIAN mask bits
EMISSION_NONE, EMISSION_DISK, EMISSION_GRID = 0, 1, 2
CMAP_AFMHOT, CMAP_GREY = 0, 1


class Sphere(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("radius", C.c_float), ("texture_id", C.c_int32), ("_pad", C.c_int32 * 3)]


class EmissionDesc(C.Structure):
    _fields_ = [
        ("index", C.c_float), ("height", C.c_float), ("r_in", C.c_float), ("r_out", C.c_float),
        ("spectral_index", C.c_float), ("absorb", C.c_float), ("gain", C.c_float), ("sense", C.c_int32),
        ("temp_power", C.c_float), ("colormap", C.c_int32), ("_pad", C.c_int32 * 2),
    ]


class PlasmaDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("lo", C.c_float * 3), ("hi", C.c_float * 3),
        ("density", C.POINTER(C.c_float)), ("temperature", C.POINTER(C.c_float)), ("velocity", C.POINTER(C.c_float)),
    ]


class FrameDesc(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("ssaa", C.c_int32), ("samples", C.c_int32),
        ("vfov", C.c_float), ("cam_pos", C.c_float * 3), ("cam_alpha", C.c_float), ("cam_beta", C.c_float),
        ("metric", C.c_int32), ("mass", C.c_float), ("spin", C.c_float),
        ("solver", C.c_int32), ("mode", C.c_int32), ("precision", C.c_int32),
        ("h", C.c_float), ("hmin", C.c_float), ("hmax", C.c_float), ("eps", C.c_float),
        ("rtol", C.c_float), ("atol", C.c_float), ("rout", C.c_float), ("horizon_eps", C.c_float),
        ("max_steps", C.c_int32), ("background_id", C.c_int32), ("bg_filter", C.c_int32), ("fxaa", C.c_int32),
        ("fp64_delta", C.c_float), ("fp64_rfac", C.c_float),
        ("nspheres", C.c_int32), ("camera", C.c_int32), ("ssaa_seed", C.c_uint32), ("emission", C.c_int32),
        ("spheres", Sphere * PRR_MAX_SPHERES),
        ("emis", EmissionDesc),
    ]

    @property
    def nrays(self) -> int:
        return self.width * self.height * self.samples


class Stats(C.Structure):
    _fields_ = [
        ("rays", C.c_int64), ("attempts", C.c_int64), ("accepted", C.c_int64), ("n_escaped", C.c_int64),
        ("n_captured", C.c_int64), ("n_intersection", C.c_int64), ("n_infinite", C.c_int64),
        ("n_math_error", C.c_int64), ("n_fp64", C.c_int64), ("kernel_ms", C.c_double), ("kernel_launches", C.c_int64),
        ("trace_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class LaunchConfig(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("blocks_per_sm", C.c_int32), ("compaction_interval", C.c_int32),
                ("rays_per_thread", C.c_int32)]


_P = C.c_void_p
_u8p = C.POINTER(C.c_uint8)
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    "prr_abi_version": (C.c_int, []),
    "prr_status_string": (C.c_char_p, [C.c_int]),
    "prr_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "prr_destroy": (None, [_P]),
    "prr_last_error": (C.c_char_p, [_P]),
    "prr_upload_texture": (C.c_int, [_P, C.c_int, _u8p, C.c_int, C.c_int]),
    "prr_upload_plasma": (C.c_int, [_P, C.POINTER(PlasmaDesc)]),
    "prr_render": (C.c_int, [_P, C.POINTER(FrameDesc), C.c_int, _u8p, _fp, C.POINTER(Stats)]),
    "prr_render_device": (C.c_int, [_P, C.POINTER(FrameDesc), C.c_int, _P, _P, _P]),
    "prr_trace_rays": (C.c_int, [_P, C.POINTER(FrameDesc), _fp, _fp, C.POINTER(Stats)]),
    "prr_trace_rays_f64": (C.c_int, [_P, C.POINTER(FrameDesc), _dp, _dp, C.POINTER(Stats)]),
    "prr_set_schedule": (C.c_int, [_P, C.c_int, C.POINTER(LaunchConfig)]),
    "prr_get_launch_config": (C.c_int, [_P, C.POINTER(LaunchConfig)]),
    "prr_autotune": (C.c_int, [_P, C.POINTER(FrameDesc), C.POINTER(LaunchConfig)]),
    "prr_set_option": (C.c_int, [_P, C.c_int, C.c_longlong]),
    "prr_measure_peak": (C.c_int, [_P, _dp, _dp]),
    "prr_check_recip": (C.c_int, [_P, _dp, C.c_int, _dp]),
    "prr_make_texture": (C.c_int, [C.c_int, C.c_uint32, C.c_int, C.c_int, _u8p]),
    "prr_frame_desc_defaults": (None, [C.POINTER(FrameDesc)]),
    "prr_sizeof": (C.c_size_t, [C.c_int]),
    "prr_adjoint": (C.c_int, [_P, C.POINTER(FrameDesc), _fp, C.c_int, _dp, C.POINTER(Stats)]),
    "prr_graph_create": (C.c_int, [_P, C.POINTER(FrameDesc), C.c_int, _P, _P, C.POINTER(_P)]),
    "prr_graph_set_frames": (C.c_int, [_P, C.POINTER(FrameDesc), C.c_int]),
    "prr_graph_launch": (C.c_int, [_P, _P]),
    "prr_graph_stats": (C.c_int, [_P, C.POINTER(Stats)]),
    "prr_graph_get_launch_config": (C.c_int, [_P, C.POINTER(LaunchConfig)]),
    "prr_graph_destroy": (None, [_P]),
    "prr_deck_load": (C.c_int, [C.c_char_p, C.POINTER(_P), C.c_char_p, C.c_size_t]),
    "prr_deck_parse_string": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
    "prr_deck_free": (None, [_P]),
    "prr_deck_has_block": (C.c_int, [_P, C.c_char_p]),
    "prr_deck_has": (C.c_int, [_P, C.c_char_p, C.c_char_p]),
    "prr_deck_get": (C.c_size_t, [_P, C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t]),
    "prr_deck_geti": (C.c_int, [_P, C.c_char_p, C.c_char_p]),
    "prr_deck_getf": (C.c_float, [_P, C.c_char_p, C.c_char_p, C.c_float]),
    "prr_deck_frame_count": (C.c_int, [_P]),
    "prr_deck_sphere_count": (C.c_int, [_P]),
    "prr_deck_sphere_texture": (C.c_size_t, [_P, C.c_int, C.c_char_p, C.c_size_t]),
    "prr_deck_frame": (C.c_int, [_P, C.c_int, C.POINTER(FrameDesc), C.c_char_p, C.c_size_t]),
    "prr_run_deck": (C.c_int, [_P, C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_int, C.POINTER(Stats)]),
    "prr_image_load": (C.c_int, [C.c_char_p, C.POINTER(_u8p), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p,
                                 C.c_size_t]),
    "prr_image_free": (None, [_u8p]),
    "prr_png_write": (C.c_int, [C.c_char_p, _u8p, C.c_int, C.c_int]),
    "prr_load_metric_plugin": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_int)]),
    "prr_render_noalloc": (C.c_int, [C.POINTER(FrameDesc), C.c_int, C.POINTER(_P), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), _P, _P, _P, C.c_char_p, C.c_size_t]),
}

_lib = None


class PrrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"prr status {status}: {message}")
        self.status = status


def load(path: str | Path | None = None) -> C.CDLL:
    """Loads the library (once) and declares every signature."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} not built: run `python -m parrelray_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def header_functions(header: Path = HEADER) -> list[str]:
    """Names of the functions include/prr.h declares."""
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(prr_[a-z0-9_]+)\s*\(", text)) - {"prr_ctx", "prr_graph", "prr_deck"})


def check(status: int, ctx=None) -> None:
    if status != OK:
        lib = load()
        msg = lib.prr_last_error(ctx).decode() if ctx else lib.prr_status_string(status).decode()
        raise PrrError(status, msg or lib.prr_status_string(status).decode())


def defaults() -> FrameDesc:
    """prr_frame_desc_defaults through the library."""
    d = FrameDesc()
    load().prr_frame_desc_defaults(C.byref(d))
    return d


def fill_defaults(d: FrameDesc) -> FrameDesc:
    """The values prr_frame_desc_defaults writes (parrelray_b200/csrc/capi.cu), set here without
    loading the library, so frame descriptors can be built where the library is not wanted (the
    CPU side of the bench).  tests/test_abi.py checks the two agree byte for byte."""
    import math

    C.memset(C.byref(d), 0, C.sizeof(d))
    d.width, d.height = 320, 180
    d.ssaa, d.samples = SSAA_NONE, 1
    d.vfov = 60.0 * math.pi / 180.0
    d.cam_pos[0] = 30.0
    d.cam_alpha, d.cam_beta = math.pi, 0.0
    d.metric, d.mass, d.spin = METRIC_SCHWARZSCHILD, 1.0, 0.0
    d.solver, d.mode, d.precision = SOLVER_RKF45, MODE_PHYSICAL, PREC_FP32
    d.h, d.hmin, d.hmax, d.eps = 0.01, 0.0001, 0.1, 0.001
    d.rtol = d.atol = 1e-6
    d.rout, d.horizon_eps, d.max_steps = 100.0, 0.001, 10000
    d.background_id, d.bg_filter, d.fxaa = -1, BG_RMS2X2, 0
    d.fp64_delta, d.fp64_rfac = 1e-3, 1.05
    d.nspheres = 0
    for i in range(PRR_MAX_SPHERES):
        d.spheres[i].texture_id = -1
    d.emission = EMISSION_NONE
    e = d.emis
    e.index, e.height, e.r_in, e.r_out = 2.0, 0.3, 2.0, 30.0
    e.spectral_index, e.absorb, e.gain, e.sense = 0.0, 0.0, 1.0, 1
    e.temp_power, e.colormap = 0.0, CMAP_AFMHOT
    return d
