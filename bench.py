"""Benchmark of the headline workload: Kerr a=0.95, 1920x1080, 2x2 SSAA
(8,294,400 rays), RKF45 at tolerance 1e-6 in FP32, three textured spheres,
2048x1024 starfield, FXAA.  One step = one full frame rendered through the
C ABI (prr_render_device: ray generation, integration, colouring, SSAA
combine, FXAA, quantisation).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 is launched with torch.distributed.run, one rank per GPU; every step
renders N frames of a camera orbit (weak scaling), the ranks pulling them
from a shared counter in the process group's store (parrelray_b200/shard.py);
NCCL carries only the barrier and the max-over-ranks time, nothing on the
data path.

Reported (one JSON line on rank 0):
  value           whole-job Mrays/s, device time (CUDA events), inputs resident
  e2e             Mrays/s through prr_render with host buffers: the frame
                  descriptor in, the 8-bit image out (pinned), copies timed
  roofline        FP32 FLOP/s of the tracing kernel: attempts x F_attempt /
                  kernel time against the measured FMA peak of the same GPU,
                  and the FP32 operations ncu counts per attempt beside it
  plain           the plain one-ray-per-thread schedule on the same GPU, with
                  the scheduler's and the geodesic form's shares of the speed-up
  accuracy        the image against an FP64 GPU render, and a seeded set of
                  the frame's rays against the FP64 host oracle
  trajectory      240 frames under one CUDA graph / per-frame / plain (all 240)
  uneven          64 uneven requests: split precision, all-FP64, all-FP32
  adjoint         one gradient of the 512x512 differentiable render
  adam_fit        200 Adam iterations of (a, i) through the adjoint
  emission        the EHT-like disk frame with and without emission
  plugin_kerr_header  the frame through the Kerr header as a metric plug-in
  cpu_baseline    the FP64 host restatement on a seeded sample of the frame's
                  rays, on this host's cores; the reference's own solver at
                  eps 1e-3 for context; the 320x180 Schwarzschild frame through
                  the reference's host build whole, beside the GPU
  reference_cuda  the reference's own CUDA build (its sources, nvcc, sm_100a)
                  on this GPU: trace_RKF at eps 1e-6 on a band of rows, and
                  its whole frame pipeline at the deck's eps 1e-3
From `plain` on, the sections run at N = 1 only: at N > 1 the line carries
the headline, e2e, roofline and stats, so that no rank waits in the final
barrier while rank 0 runs single-GPU studies.
`--impl reference` runs the CPU arm alone: the FP64 host restatement on a
fixed seeded sample of the frame's rays each step (see run_reference_arm).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "Mrays/s, Kerr a=0.95 1080p: plain vs batched FP32 at ≤1/255 err; adjoint ms"
WORKLOAD = "kerr_a0.95_1920x1080_ssaa2x2_fxaa_rkf45_tol1e-6_fp32_3spheres"

# Algorithmic FP32 work of one RKF45 attempt (FMA = 2 flop; sqrt, division,
# reciprocal, pow = 1).  Stage combinations of the reference's formulation
# (kernels/solver.cuh:163-176: 12 stage vectors, two 6-term sums for each of
# x and u at 4th and 5th order, error max, step update) = 492; the Kerr
# geodesic acceleration in the Kerr-Schild contraction form
# (parrelray_b200/csrc/prr_device.cuh:geod_ks) = 168 per evaluation, 6 per
# attempt.  Sphere tests are not counted.
FLOPS_STAGES = 492
FLOPS_GEOD_KERR = 168
F_ATTEMPT = 6 * FLOPS_GEOD_KERR + FLOPS_STAGES

# FP32 operations the tracing kernels actually execute per attempt, from ncu's instruction counters on
# the 960x540 copy of the headline frame (one launch, 64-thread CTAs at 8 per SM, refill every 64
# attempts): FFMA x 2 FLOP, paired FFMA2 x 4 (two FMAs per thread instruction), FMUL/FADD x 1, paired
# FMUL2/FADD2 x 2, summed and divided by the launch's attempt counter.  k_ham (the Hamiltonian form)
# executes 938 FLOP per attempt; k_pair (the (x, u) contraction, the form F_ATTEMPT counts) 1,459.
NCU_FLOP_PER_ATTEMPT = {"k_ham": 938.0, "k_pair": 1459.0}
NCU_FLOP_RULE = ("FP32 FLOP executed, from ncu sass_thread_inst_executed_op_{ffma,fmul,fadd}{,2}: FFMA 2, FFMA2 4, "
                 "FMUL/FADD 1, FMUL2/FADD2 2, per attempt")
# DRAM bytes of one launch of the tracing kernel (ncu, 960x540 copy of the headline frame)
TRAFFIC_PER_LAUNCH = 8.724224e6


def reserve_stdout():
    """Points file descriptor 1 at stderr for the rest of the run and returns
    a stream on the original stdout: the result line is then the only line on
    stdout, whatever the reference host build (whose solver prints with printf)
    or a library writes."""
    sys.stdout.flush()
    fd = os.dup(1)
    os.dup2(2, 1)
    sys.stdout = sys.stderr
    return os.fdopen(fd, "w", buffering=1)


RESULT_OUT = sys.stdout


def emit(line: dict) -> None:
    print(json.dumps(line), file=RESULT_OUT, flush=True)


def pair_kernel_name(cfg) -> str:
    """The FP32 renderer instantiation a launch shape selects (k_persistent.cu: launch_persistent; one
    pixel per thread: the Hamiltonian-form k_ham, two: k_pair)."""
    if cfg.rays_per_thread == 2:
        return "k_pair<2,256,1>"
    return "k_ham<64,8>" if cfg.block_size <= 64 else "k_ham<256,1>"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def quantize(img: np.ndarray) -> np.ndarray:
    """roundf(255 x) of the clamped float colour (cudamaths/image.cu:31)."""
    v = np.float32(255.0) * np.clip(img.astype(np.float32), np.float32(0.0), np.float32(1.0))
    return np.floor(v.astype(np.float64) + 0.5).astype(np.uint8)


def pixel_rule(a8: np.ndarray, b8: np.ndarray) -> float:
    """Fraction of pixels whose RGB differ by at most 1/255 in every channel."""
    d = np.abs(a8.astype(np.int32) - b8.astype(np.int32)).max(axis=-1)
    return float(np.mean(d <= 1))


def orbit_frames(world: int, width: int, height: int) -> list:
    """The frames of one step: one per rank, frame k with the spheres advanced k/world of an orbit
    (frame 0 is the headline frame)."""
    from parrelray_b200 import scenes

    frames = []
    for k in range(world):
        d = scenes.kerr_1080p_ssaa4(width, height)
        ang = 2 * math.pi * k / world
        for j in range(d.nspheres):
            sp = d.spheres[j]
            x, y = sp.center[0], sp.center[1]
            sp.center[0] = scenes.f32(x * math.cos(ang) - y * math.sin(ang))
            sp.center[1] = scenes.f32(x * math.sin(ang) + y * math.cos(ang))
        frames.append(d)
    return frames


def workload_config(width: int, height: int) -> dict:
    """The `config` object of both arms' result lines (the workload, nothing arm-specific)."""
    return {"workload": WORKLOAD, "rays_per_step": width * height * 4, "width": width, "height": height,
            "samples": 4, "tolerance": 1e-6, "metric": "kerr a=0.95 M=1", "camera": "r=25M i=80deg fov=50deg",
            "l2": "GPU arm: a 256 MiB buffer (L2 is 126 MB) is written between timed steps; CPU arm: no GPU"}


def mapped_repo_libraries() -> list[str]:
    """The repository's shared libraries mapped into this process (from /proc/self/maps)."""
    out = set()
    try:
        for line in Path("/proc/self/maps").read_text().splitlines():
            path = line.split()[-1] if line.split() else ""
            if path.endswith(".so") and path.startswith(str(REPO)):
                out.add(str(Path(path).relative_to(REPO)))
    except OSError:
        pass
    return sorted(out)


def oracle_fp64_sample(orc, frame64, textures, ids, nthreads: int) -> dict:
    """The FP64 PHYSICAL host restatement (oracle/prr_oracle.cpp: Christoffel-table geodesic, atol/rtol
    control at the frame's tolerance) on the rays `ids` of `frame64`, all `nthreads` host threads."""
    t0 = time.perf_counter()
    st, _ = orc.trace(frame64, textures, precision=1, ids=ids, nthreads=nthreads)
    secs = time.perf_counter() - t0
    return {"rays": int(len(ids)), "seconds": secs, "mrays_s": len(ids) / secs / 1e6,
            "results": np.bincount(st[:, 2].astype(int), minlength=5).tolist()}


def calibrated_ray_sample(orc, frame64, textures, target_s: float, nthreads: int, seed: int = 2024,
                          lo: int = 1024, hi: int = 262144) -> np.ndarray:
    """A seeded uniform sample of the frame's rays sized so the FP64 oracle traces it in about
    `target_s` seconds on `nthreads` threads (a multiple of 1024 rays in [lo, hi]); the sample is
    an unbiased estimate of the whole frame's per-ray cost."""
    order = np.random.default_rng(seed).permutation(frame64.nrays)
    probe = oracle_fp64_sample(orc, frame64, textures, np.sort(order[:lo]), nthreads)
    n = int(min(max(round(probe["mrays_s"] * 1e6 * target_s / lo) * lo, lo), hi))
    return np.sort(order[:n])


def cpu_reference_sample(frame, textures, budget_s: float, nthreads: int, eps: float):
    """The reference's own solver (its sources built for the host, oracle/_ref, with the Kerr-Schild
    plug-in header) on a bounded sample of `frame`'s rays: 8-ray blocks in a fixed pseudo-random
    order until `budget_s` of wall time is spent.  `eps` is the reference's absolute error tolerance."""
    from oracles import RefHost, ref_available, write_deck

    from parrelray_b200 import abi, scenes

    if not ref_available("kerr"):
        return None
    ref_frame = scenes.kerr_1080p_ssaa4(frame.width, frame.height, mode=abi.MODE_REFERENCE, eps=eps,
                                        horizon_eps=0.001)
    _, a_deg, b_deg = scenes.camera_pose(25.0, 80.0)
    deck = write_deck(Path("/tmp/prrbench"), ref_frame, textures, fov_deg=50.0, a_deg=a_deg, b_deg=b_deg)
    ref = RefHost("kerr")
    assert ref.load(deck) == 1
    ref.prepare(0, nthreads)
    nbx = frame.samples * frame.width // 8
    rng = np.random.default_rng(7)
    order = rng.permutation(nbx * frame.height)[:4096]
    done, secs = 0, 0.0
    chunk = max(nthreads, 1)
    while done < len(order) and secs < budget_s:
        sel = order[done:done + chunk]
        secs += ref.trace_blocks(sel % nbx, sel // nbx, nthreads)
        done += len(sel)
    rays = done * 8
    results = np.array([ref.lib.prr_ref_ray_result(int((r * frame.width * frame.samples) + 8 * b + t))
                        for b, r in zip(order[:done] % nbx, order[:done] // nbx) for t in range(8)])
    return {"rays": rays, "seconds": secs, "mrays_s": rays / secs / 1e6 if secs > 0 else None, "eps": eps,
            "infinite_geo_fraction": float(np.mean(results == abi.RESULT_INFINITE_GEO)) if len(results) else None}


def single_frame_workload(ctx, nthreads: int) -> dict:
    """The single-frame Schwarzschild workload (M = 1, camera r = 30M, inclination 85 deg, FOV 60 deg,
    320x180, one sphere R = 1M at r = 10M, the standard textures), the frame the reference's host
    build can render whole in seconds: its own solver on all host threads at the deck's eps = 1e-3
    (prr.cpp:237-341: ray placement, initRays, trace_RKF, rayToRGB, combineSamples), beside this
    library's REFERENCE mode on the GPU (same algorithm, quirks and eps) and its PHYSICAL FP32 render
    at the workload's tolerance 1e-6 (stop at r <= 2.01M)."""
    from oracles import RefHost, ref_available, write_deck

    from parrelray_b200 import abi, scenes

    tex = scenes.standard_textures()
    ctx.upload_textures(tex)
    ref_mode = scenes.schwarzschild_320(mode=abi.MODE_REFERENCE, eps=1e-3, horizon_eps=0.001)
    phys = scenes.schwarzschild_320(horizon_eps=0.01)
    res = {"workload": "schwarzschild_320: M=1, r=30M, i=85 deg, FOV 60 deg, 320x180, 1 sphere, 57,600 rays"}
    ctx.render(ref_mode)
    g8, _, gst = ctx.render(ref_mode)
    ctx.render(phys)
    _, _, pst = ctx.render(phys)
    res["gpu_reference_mode_eps_1e-3"] = {"ms": gst.kernel_ms, "mrays_s": gst.rays / (gst.kernel_ms * 1e-3) / 1e6}
    res["gpu_physical_fp32_tol_1e-6"] = {"ms": pst.kernel_ms, "mrays_s": pst.rays / (pst.kernel_ms * 1e-3) / 1e6,
                                         "infinite_geo": int(pst.n_infinite)}
    if ref_available("schw"):
        _, a_deg, b_deg = scenes.camera_pose(30.0, 85.0)
        deck = write_deck(Path("/tmp/prrbench320"), ref_mode, tex, fov_deg=60.0, a_deg=a_deg, b_deg=b_deg)
        ref = RefHost("schw")
        assert ref.load(deck) == 1
        out = ref.frame(0, nthreads)
        res["reference_host_eps_1e-3"] = {"seconds": out["seconds"], "threads": nthreads,
                                          "mrays_s": ref_mode.nrays / out["seconds"] / 1e6,
                                          "what": "the reference's frame pipeline (its sources built for the host, "
                                                  "OpenMP over its 8x8 blocks) on the whole frame"}
        res["gpu_reference_mode_vs_reference_host"] = {
            "speedup": out["seconds"] / (gst.kernel_ms * 1e-3),
            "pixels_within_1_255": pixel_rule(g8[0], quantize(out["image"]))}
    return res


def bench_reference_cuda(width: int, height: int, timeout_s: float = 240.0):
    """The reference's own CUDA build on this GPU, in a child process (the reference ends its process
    on any CUDA error, prr.cpp:37-47, and resets the device): see reference_cuda_child."""
    import tempfile

    with tempfile.TemporaryDirectory() as td:
        out = Path(td) / "refcuda.json"
        try:
            r = subprocess.run([sys.executable, str(Path(__file__).resolve()), "--refcuda-child", str(out),
                                "--width", str(width), "--height", str(height)],
                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=timeout_s)
        except subprocess.TimeoutExpired:
            return {"unavailable": f"the reference CUDA run did not finish in {timeout_s:.0f} s"}
        if r.returncode != 0 or not out.exists():
            return {"unavailable": f"the reference CUDA run exited with status {r.returncode}"}
        return json.loads(out.read_text())


def reference_cuda_child(out_path: str, width: int, height: int, nlines: int = 4) -> int:
    """oracle/_ref/libprr_refcu_kerr.so: the reference's sources compiled with nvcc for sm_100a, the
    Kerr plug-in header, its <<<>>> launches.  trace_RKF at the workload's eps = 1e-6 on the band of
    `nlines` rows at the middle of the frame (through the shadow; at this tolerance most rays run to
    the 1e6-attempt cap, so the whole frame would take minutes), then its frame pipeline renderframe
    (prr.cpp:237-341, PNG save included) at the deck's eps = 1e-3.  Writes a JSON object."""
    import ctypes as C

    sys.path.insert(0, str(REPO / "tests"))
    from oracles import write_deck

    from parrelray_b200 import abi, scenes

    frame = scenes.kerr_1080p_ssaa4(width, height)
    textures = scenes.standard_textures()
    layer = max(height // 2 - nlines, 0) // nlines  # rows 536-539 of 1080

    path = REPO / "oracle" / "_ref" / "libprr_refcu_kerr.so"
    if not path.exists():
        Path(out_path).write_text(json.dumps({"unavailable": "reference CUDA build (oracle/_ref/libprr_refcu_kerr.so) not built"}))
        return 0
    lib = C.CDLL(str(path))
    lib.prr_refcu_load.restype = C.c_int
    lib.prr_refcu_load.argtypes = [C.c_char_p]
    lib.prr_refcu_trace_rows.restype = C.c_double
    lib.prr_refcu_trace_rows.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
    lib.prr_refcu_render.restype = C.c_double
    lib.prr_refcu_render.argtypes = [C.c_int, C.POINTER(C.c_float)]
    lib.prr_refcu_set_eps.restype = None
    lib.prr_refcu_set_eps.argtypes = [C.c_float]
    ref_frame = scenes.kerr_1080p_ssaa4(frame.width, frame.height, mode=abi.MODE_REFERENCE, eps=1e-6,
                                        horizon_eps=0.001)
    _, a_deg, b_deg = scenes.camera_pose(25.0, 80.0)
    deck = write_deck(Path("/tmp/prrbenchrefcu"), ref_frame, textures, fov_deg=50.0, a_deg=a_deg, b_deg=b_deg)
    nf = lib.prr_refcu_load(str(deck).encode())
    if nf != 1:
        Path(out_path).write_text(json.dumps({"unavailable": f"prr_refcu_load returned {nf}"}))
        return 0
    layers = np.array([layer], dtype=np.int32)
    counts = np.zeros(5, dtype=np.int64)
    ms = lib.prr_refcu_trace_rows(0, nlines, 1, layers.ctypes.data_as(C.POINTER(C.c_int)),
                                  counts.ctypes.data_as(C.POINTER(C.c_longlong)))
    if ms < 0:
        Path(out_path).write_text(json.dumps({"unavailable": "prr_refcu_trace_rows failed"}))
        return 0
    rays = int(counts.sum())
    res = {"what": "the reference's own kernels (kernels/solver.cuh trace_RKF, 8x8 blocks, one ray per thread) "
                   "built with nvcc for sm_100a, Kerr-Schild plug-in header",
           "eps_1e-6_sample": {"rows": f"{layer * nlines}-{(layer + 1) * nlines - 1}", "rays": rays, "ms": ms,
                               "mrays_s": rays / (ms * 1e-3) / 1e6,
                               "infinite_geo_fraction": float(counts[abi.RESULT_INFINITE_GEO] / max(rays, 1))}}
    lib.prr_refcu_set_eps(1e-3)
    img = np.zeros((frame.height, frame.width, 3), dtype=np.float32)
    secs = lib.prr_refcu_render(0, img.ctypes.data_as(C.POINTER(C.c_float)))
    if secs > 0:
        res["eps_1e-3_frame"] = {"seconds": secs, "mrays_s": frame.nrays / secs / 1e6,
                                 "what": "renderframe at the deck's default tolerance (not the workload's 1e-6), "
                                         "wall time of its launches, synchronisations and PNG save",
                                 "black_pixel_fraction": float(np.mean(img.max(axis=-1) <= 0.0))}
    Path(out_path).write_text(json.dumps(res))
    return 0


def bench_trajectory(ctx, torch, stream, plain_stride: int = 1):
    """The 240-frame trajectory workload: Kerr a = 0.9, 960x540, no SSAA,
    orbit radius 20M -> 8M, inclination 60 -> 88 deg, tolerance 1e-6, FP32.
    (1) autotuned launch shape, whole trajectory recorded into one CUDA graph
    and replayed (one persistent launch); (2) the same frames as 240
    persistent launches, one per frame; (3) the plain one-ray-per-thread
    schedule, one render call per frame, on every frame (`plain_stride` > 1
    renders every n-th frame and scales by rays)."""
    from parrelray_b200 import Graph, abi, scenes

    frames = scenes.trajectory_240()
    npx = sum(f.width * f.height for f in frames)
    rays = sum(f.nrays for f in frames)
    out8 = torch.empty(npx * 3, dtype=torch.uint8, device="cuda")
    saved = ctx.launch_config()
    t0 = time.perf_counter()
    tuned = ctx.autotune(frames[len(frames) // 2])
    tune_s = time.perf_counter() - t0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = {"workload": "trajectory_240: Kerr a=0.9, 240 frames 960x540, r 20M->8M, i 60->88 deg, tol 1e-6, FP32",
           "rays": rays, "autotune_s": tune_s,
           "tuned": {"block_size": tuned.block_size, "blocks_per_sm": tuned.blocks_per_sm,
                     "compaction_interval": tuned.compaction_interval, "rays_per_thread": tuned.rays_per_thread}}
    with Graph(ctx, frames, out8.data_ptr()) as g:
        g.launch(stream.cuda_stream)  # warm-up replay
        st = g.stats()
        ev0.record(stream)
        g.launch(stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        graph_ms = ev0.elapsed_time(ev1)
    res["graph"] = {"ms": graph_ms, "mrays_s": rays / (graph_ms * 1e-3) / 1e6, "launches": int(st.kernel_launches),
                    "attempts": int(st.attempts)}
    # one persistent launch per frame (same tuned shape), no graph
    ev0.record(stream)
    for f in frames:
        ctx.render_device(f, out8.data_ptr(), stream=stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    pf_ms = ev0.elapsed_time(ev1)
    res["per_frame_persistent"] = {"ms": pf_ms, "mrays_s": rays / (pf_ms * 1e-3) / 1e6, "launches": len(frames)}
    ctx.set_schedule(abi.SCHED_PERSISTENT, saved)
    # plain schedule, one render call per frame, sampled
    ctx.set_schedule(abi.SCHED_PLAIN)
    sample = frames[::plain_stride]
    ctx.render_device(sample[0], out8.data_ptr(), stream=stream.cuda_stream)  # warm-up
    ev0.record(stream)
    for f in sample:
        ctx.render_device(f, out8.data_ptr(), stream=stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    ctx.set_schedule(abi.SCHED_PERSISTENT, saved)
    plain_sample_ms = ev0.elapsed_time(ev1)
    sample_rays = sum(f.nrays for f in sample)
    plain_rate = sample_rays / (plain_sample_ms * 1e-3) / 1e6
    if plain_stride == 1:
        res["plain_per_frame"] = {"ms": plain_sample_ms, "mrays_s": plain_rate, "frames": len(sample),
                                  "what": "every frame rendered with the plain schedule, one call per frame"}
    else:
        res["plain_per_frame"] = {"mrays_s": plain_rate, "ms_240_estimated": rays / (plain_rate * 1e6) * 1e3,
                                  "sampled_frames": len(sample), "sampled_ms": plain_sample_ms,
                                  "what": f"every {plain_stride}th frame rendered with the plain schedule, one call "
                                          f"per frame; time scaled to the 240 frames by rays"}
    res["speedup_vs_plain"] = res["graph"]["mrays_s"] / plain_rate
    res["speedup_vs_per_frame_persistent"] = pf_ms / graph_ms
    return res


def bench_emission(ctx, torch, stream, size: int = 1024, reps: int = 3):
    """Plasma emission: the EHT-like frame (Kerr a = 0.94, i = 17 deg, pinhole
    camera, thick co-rotating disk, r_+ .. 20M) at size x size with 2x2 SSAA,
    FP32, tolerance 1e-6, timed with CUDA events around `reps` renders; the
    same frame with emission off (the cost of the emission hook); FP32 vs FP64
    at 256x256 (pixels within 1/255)."""
    from parrelray_b200 import abi, scenes

    f = scenes.eht_disk(size, samples=4)
    off = scenes.eht_disk(size, samples=4)
    off.emission = abi.EMISSION_NONE
    out8 = torch.empty(size * size * 3, dtype=torch.uint8, device="cuda")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = {"workload": f"eht_disk: Kerr a=0.94, i=17 deg, r=50M, pinhole FOV 27 deg, {size}x{size}, 2x2 SSAA, "
                       "thick disk n ~ r^-3, FP32, tol 1e-6", "rays": f.nrays}
    for name, fr in (("emission", f), ("no_emission", off)):
        ctx.render_device(fr, out8.data_ptr(), stream=stream.cuda_stream)  # warm-up
        ev0.record(stream)
        for _ in range(reps):
            ctx.render_device(fr, out8.data_ptr(), stream=stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / reps
        res[name] = {"ms": ms, "mrays_s": fr.nrays / (ms * 1e-3) / 1e6}
    st = ctx.render(f)[2]
    res["emission"]["accepted_steps"] = int(st.accepted)
    res["emission_overhead"] = res["emission"]["ms"] / res["no_emission"]["ms"]
    a = ctx.render(scenes.eht_disk(256, samples=4))[0][0].astype(np.int32)
    b = ctx.render(scenes.eht_disk(256, samples=4, precision=abi.PREC_FP64))[0][0].astype(np.int32)
    d = np.abs(a - b).max(axis=-1)
    res["fp32_vs_fp64_256"] = {"pixels_within_1_255": float(np.mean(d <= 1)), "max_abs_diff_255": int(d.max())}
    return res


def bench_uneven(ctx, torch, stream, textures, oracle_rays_per_request: int = 64, oracle_seconds: float = 10.0):
    """The 64-request workload (log-uniform 256x256..2048x1024, a ~ U[0, 0.998],
    r ~ U[8M, 40M], i ~ U[10, 89] deg, tolerance 1e-7) in one batched render
    per precision: SPLIT (FP32 bulk, FP64 re-integration near the critical
    impact parameter or the horizon), all-FP64 and plain FP32.  Per request:
    fraction of pixels within 1/255 of the all-FP64 GPU render, and the
    per-sample colour error of the SPLIT render against the FP64 host oracle
    on a seeded sample of rays (no SSAA, so a sample is a pixel)."""
    from parrelray_b200 import abi, scenes

    res = {"workload": "uneven_64: 64 requests, log-uniform 256^2..2048x1024, a~U[0,0.998], r~U[8,40]M, "
                       "i~U[10,89] deg, tol 1e-7"}
    imgs, stats, ms = {}, {}, {}
    for name, p in (("split", abi.PREC_SPLIT), ("fp64", abi.PREC_FP64), ("fp32", abi.PREC_FP32)):
        fr = scenes.uneven_64(precision=p)
        im, _, st = ctx.render(fr)
        imgs[name], stats[name], ms[name] = im, st, st.trace_ms
    rays = int(stats["split"].rays)
    res["rays"] = rays
    for name in ms:
        res[name] = {"ms": ms[name], "mrays_s": rays / (ms[name] * 1e-3) / 1e6,
                     "render_call_ms": stats[name].kernel_ms, "attempts": int(stats[name].attempts)}
    res["timing"] = "ms = tracing kernels (persistent pass, plus the FP64 pass for SPLIT), CUDA events; " \
                    "render_call_ms adds combine/quantise and the first-call buffer growth"
    res["split"]["fp64_rays"] = int(stats["split"].n_fp64)
    res["speedup_split_vs_fp64"] = ms["fp64"] / ms["split"]
    per = []
    for a, b in zip(imgs["split"], imgs["fp64"]):
        d = np.abs(a.astype(np.int32) - b.astype(np.int32)).max(axis=-1)
        per.append(float(np.mean(d <= 1)))
    per32 = []
    for a, b in zip(imgs["fp32"], imgs["fp64"]):
        d = np.abs(a.astype(np.int32) - b.astype(np.int32)).max(axis=-1)
        per32.append(float(np.mean(d <= 1)))
    tot = sum(a.shape[0] * a.shape[1] for a in imgs["fp64"])
    res["vs_fp64_gpu"] = {"min_request_fraction_within_1_255": min(per),
                          "all_pixels_fraction_within_1_255": sum(p * a.shape[0] * a.shape[1]
                                                                  for p, a in zip(per, imgs["fp64"])) / tot,
                          "per_request": [round(p, 6) for p in per],
                          "fp32_min_request_fraction": min(per32),
                          "fp32_all_pixels_fraction": sum(p * a.shape[0] * a.shape[1]
                                                          for p, a in zip(per32, imgs["fp64"])) / tot}
    # FP64 host oracle on a bounded seeded sample of rays of every request
    try:
        sys.path.insert(0, str(REPO / "tests"))
        from oracles import Oracle

        orc = Oracle()
    except (ImportError, FileNotFoundError):
        return res
    fr64 = scenes.uneven_64(precision=abi.PREC_FP64)
    rng = np.random.default_rng(11)
    errs, n_done, t0 = [], 0, time.perf_counter()
    for k, f in enumerate(fr64):
        if time.perf_counter() - t0 > oracle_seconds:
            break
        ids = rng.choice(f.nrays, size=min(oracle_rays_per_request, f.nrays), replace=False)
        _, rgb = orc.trace(f, textures, precision=1, ids=ids)
        img = imgs["split"][k].reshape(-1, 3).astype(np.int32)
        q = np.floor(np.float32(255.0) * np.clip(rgb, 0, 1).astype(np.float32) + 0.5).astype(np.int32)
        errs.append(np.abs(img[ids] - q).max(axis=-1))
        n_done += 1
    e = np.concatenate(errs) if errs else np.zeros(0)
    res["vs_fp64_host_oracle"] = {"requests": n_done, "rays": int(e.size),
                                  "fraction_within_1_255": float(np.mean(e <= 1)) if e.size else None,
                                  "max_diff_255": int(e.max()) if e.size else None}
    return res


def smooth_sky(w: int = 512, h: int = 256) -> np.ndarray:
    """A low-frequency RGBA8 sky: with it the image is a smooth function of the camera, so the L2
    inverse problem is well posed (a point-star sky makes the loss nearly random in the inclination)."""
    x = np.arange(w)[None, :]
    y = np.arange(h)[:, None]
    t = np.zeros((h, w, 4), np.uint8)
    t[..., 0] = (128 + 90 * np.sin(2 * np.pi * x / w) * np.ones_like(y)).astype(np.uint8)
    t[..., 1] = (128 + 90 * np.cos(np.pi * y / h) * np.ones_like(x)).astype(np.uint8)
    t[..., 2] = (128 + 60 * np.sin(4 * np.pi * x / w + 2 * np.pi * y / h)).astype(np.uint8)
    t[..., 3] = 255
    return t


def adjoint_diagnosis(ctx, size: int, extra: dict, h: float = 1e-3, margin: int = 2) -> dict:
    """At the fit's start (a = 0.3, i = 45 deg; FP64 renders and adjoint) and for the linearised loss
    sum(w * image), w = 2 (image - target): the adjoint gradient against central differences of the
    renders at +-h (weights held fixed), (1) over all pixels, (2) over the pixels whose discrete events
    (result and accepted-step count of the ray, from prr_trace_rays_f64) are the same at -h, 0 and +h,
    and (3) over the fit's sky weights (inverse.sky_weights with `margin`).  The adjoint freezes those
    events, so it is the derivative of (2); (1) also carries the silhouette pixels, whose ray switches
    between sky and shadow inside +-h or winds near the photon orbit."""
    from parrelray_b200 import abi, inverse, scenes

    def frame(a, incl):
        return scenes.kerr_512_adjoint(spin=a, incl_deg=incl, precision=abi.PREC_FP64, size=size, **extra)

    def image(d):
        return ctx.render(d, want_float=True)[1][0].astype(np.float64)

    def signature(d):
        st = ctx.trace_rays_f64(d)[0]
        return (st[:, 2].astype(np.int64) * 1000003 + st[:, 11].astype(np.int64)).reshape(d.height, d.width)

    def adjoint(d, w):
        return ctx.adjoint(d, w)[0]

    tgt = image(frame(0.7, 60.0))
    d0 = frame(0.3, 45.0)
    img0 = image(d0)
    w = 2.0 * (img0 - tgt)
    sky = inverse.sky_weights(img0, tgt, margin)[:, :, None]
    s0 = signature(d0)
    g_all = adjoint(d0, w)
    g_sky = adjoint(d0, w * sky)
    out = {}
    hd = math.degrees(h)
    for name, k, (dp, dm) in (("spin", 0, (frame(0.3 + h, 45.0), frame(0.3 - h, 45.0))),
                              ("inclination", 2, (frame(0.3, 45.0 + hd), frame(0.3, 45.0 - hd)))):
        ip, im = image(dp), image(dm)
        same = (signature(dp) == s0) & (signature(dm) == s0)
        fd_all = float(np.sum(w * (ip - im)) / (2 * h))
        fd_same = float(np.sum(w * same[:, :, None] * (ip - im)) / (2 * h))
        fd_sky = float(np.sum(w * sky * (ip - im)) / (2 * h))
        g_same = adjoint(d0, w * same[:, :, None])
        out[name] = {"adjoint_all_pixels": float(g_all[k]), "central_difference_all_pixels": fd_all,
                     "adjoint_same_events": float(g_same[k]), "central_difference_same_events": fd_same,
                     "adjoint_sky_weights": float(g_sky[k]), "central_difference_sky_weights": fd_sky,
                     "pixels_with_event_changes": float(1.0 - same.mean())}
    out["sky_weight_fraction"] = float(sky.mean())
    out["what"] = ("h = 1e-3 (spin; inclination in radians); the adjoint equals the central difference over "
                   "pixels whose events do not change and over the sky weights; over all pixels the silhouette "
                   "decides the sign of the spin derivative, which is why the fit weights the loss")
    return out


def bench_adam_fit(ctx, iters: int, size: int, lr: float = 0.01, decay: float = 0.99, sphere: bool = False,
                   margin: int = 2):
    """The inverse problem of the differentiable-render workload: target rendered at a = 0.7,
    inclination 60 deg (camera r = 20M, sphere phase 30 deg); Adam on (a, inclination) from (0.3,
    45 deg) with the step decaying as lr * decay^t, every gradient from prr_adjoint on the FP32
    render (FP32 forward steps, FP64 adjoint and reduction), the loss restricted to the pixels that
    show sky in both images at least `margin` pixels from the shadow (inverse.sky_weights).  Smooth
    sky (see smooth_sky)."""
    from parrelray_b200 import abi, inverse, scenes

    ctx.upload_texture(scenes.SKY_ID, smooth_sky())
    extra = {} if sphere else {"spheres": []}
    diagnosis = adjoint_diagnosis(ctx, size, extra, margin=margin)

    def frame_at(q):
        return scenes.kerr_512_adjoint(spin=float(q[0]), incl_deg=math.degrees(q[1]), precision=abi.PREC_FP32,
                                       size=size, **extra)

    _, tgt, _ = ctx.render(frame_at((0.7, math.radians(60.0))), want_float=True)
    h = inverse.fit(ctx, frame_at, tgt[0], (0.3, math.radians(45.0)), (0, 2), iters, lr, decay, margin,
                    0 if sphere else -1, lo=(0.0, 0.0), hi=(0.99, math.pi))
    ctx.upload_textures(scenes.standard_textures())
    loss = h["loss"]
    qf = h["q_final"]
    return {"workload": f"Adam on (a, i) from (0.3, 45 deg) towards (0.7, 60 deg), {size}x{size}, FP32 forward / "
                        f"FP64 adjoint, smooth sky" + ("" if sphere else ", no sphere"),
            "loss": f"L2 over the pixels that show sky in both images, >= {margin} px from a shadow pixel of either",
            "iterations": iters, "lr": lr, "lr_decay": decay,
            "loss_first": loss[0], "loss_last": loss[-1], "loss_min": min(loss),
            "weighted_loss_first": h["weighted_loss"][0], "weighted_loss_last": h["weighted_loss"][-1],
            "weighted_fraction_first_last": [h["weighted_fraction"][0], h["weighted_fraction"][-1]],
            "a_final": float(qf[0]), "incl_final_deg": math.degrees(qf[1]),
            "error_final": {"spin": float(qf[0]) - 0.7, "inclination_deg": math.degrees(qf[1]) - 60.0},
            "device_ms_per_iteration": float(np.mean(h["device_ms"])), "wall_s": h["wall_s"],
            "losses_every_20": [round(x, 4) for x in loss[::20]],
            "gradient_at_start": diagnosis}


def run_reference_arm(args):
    """The CPU arm: the headline frame's rays through the FP64 PHYSICAL host restatement
    (oracle/prr_oracle.cpp) at the workload's tolerance 1e-6 on all host threads - the reference has
    no Kerr solver of its own (its metrics/kerr.cuh returns a zero geodesic), and its FP32
    absolute-error solver with the Kerr plug-in header sends most rays to its iteration cap at this
    tolerance, so the restatement stands in for it.  Every step traces the same seeded uniform
    sample of the frame's rays, sized so a step takes about PRR_REF_STEP_SECONDS (default 4);
    `value` is rays per second over the timed steps and `ms_per_step` the measured step time.  The
    reference's own solver (host build) on the same frame at eps 1e-3, where its error test still
    works, is reported beside it for context.  Loads no library of the product."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, str(REPO / "tests"))
    try:
        from oracles import Oracle

        orc = Oracle()
    except (ImportError, FileNotFoundError) as e:
        emit({"impl": "reference", "unavailable": f"the CPU oracle library is not built ({e})"})
        return 0
    from parrelray_b200 import abi, scenes

    nthreads = os.cpu_count() or 1
    tex = orc.standard_textures()
    frame64 = scenes.kerr_1080p_ssaa4(args.width, args.height, precision=abi.PREC_FP64)
    target = float(os.environ.get("PRR_REF_STEP_SECONDS", "4"))
    ids = calibrated_ray_sample(orc, frame64, tex, target, nthreads)
    times, results = [], None
    for it in range(args.warmup + args.steps):
        r = oracle_fp64_sample(orc, frame64, tex, ids, nthreads)
        if it >= args.warmup:
            times.append(r["seconds"])
            results = r["results"]
    secs = float(np.sum(times))
    mr = len(ids) * len(times) / secs / 1e6
    ms_per_step = 1e3 * secs / len(times)
    context = cpu_reference_sample(frame64, tex, 4.0, nthreads, eps=1e-3)
    sample = (f"{len(ids)} rays drawn uniformly (seed 2024) from the {frame64.nrays}-ray frame, the same rays "
              f"every step, FP64 PHYSICAL restatement at tolerance 1e-6, {nthreads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": mr, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded procedural textures)",
        "config": workload_config(args.width, args.height),
        "cpu_baseline": {"value": mr, "unit": "Mrays/s", "cores": nthreads, "kind": "port", "sample": sample,
                         "results": {"success": results[abi.RESULT_SUCCESS],
                                     "intersection": results[abi.RESULT_INTERSECTION],
                                     "infinite_geo": results[abi.RESULT_INFINITE_GEO],
                                     "math_error": results[abi.RESULT_MATH_ERROR]},
                         "reference_solver_eps_1e-3": dict(context, what=(
                             "the reference's own trace_RKF (its sources built for the host, Kerr-Schild plug-in "
                             "header) on 8-ray blocks across the frame at the deck's default eps 1e-3 - context "
                             "only: a looser tolerance than the workload's")) if context else None},
        "e2e": {"value": mr, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "libraries_loaded": mapped_repo_libraries(),
    }
    emit(line)
    return 0


def bench_plugin_kerr(ctx, torch, stream, frame) -> dict:
    """The headline frame through the Kerr header shipped as a metric plug-in (compat/metrics/kerr.cuh:
    the geodesic by the full Christoffel table, as a plug-in author writes it) in PHYSICAL FP32 mode on
    the persistent scheduler, beside the built-in metric; pixels within 1/255 of each other."""
    from parrelray_b200 import abi

    p = REPO / "parrelray_b200" / "_lib" / "libprr_metric_kerr.so"
    if not p.exists():
        return {"unavailable": "libprr_metric_kerr.so not built"}
    d = abi.FrameDesc.from_buffer_copy(frame)
    d.horizon_eps = 0.001  # the header's User_ENDLOOP stops at r_+ + 0.001
    d.metric = ctx.load_metric_plugin(p)
    ctx.render(d)
    img, _, st = ctx.render(d)
    b = abi.FrameDesc.from_buffer_copy(frame)
    b.horizon_eps = 0.001
    bimg, _, bst = ctx.render(b)
    return {"plugin_ms": st.kernel_ms, "plugin_mrays_s": st.rays / (st.kernel_ms * 1e-3) / 1e6,
            "builtin_ms": bst.kernel_ms, "builtin_mrays_s": bst.rays / (bst.kernel_ms * 1e-3) / 1e6,
            "builtin_speedup": st.kernel_ms / bst.kernel_ms, "plugin_attempts": int(st.attempts),
            "pixels_within_1_255": pixel_rule(img[0], bimg[0]),
            "what": "the same 1080p frame, PHYSICAL FP32, through the shipped Kerr plug-in header (Christoffel "
                    "table, persistent plug-in kernel + the header's rayToRGB) and through the built-in metric"}


def bench_accuracy(ctx, frame, fp64_peak, n_oracle_rays: int = 4096) -> dict:
    """The headline frame against FP64: (1) the whole image against an FP64 render of the same frame on
    the GPU; (2) a fixed seeded set of the frame's rays traced by the FP64 host oracle (the checker,
    Christoffel-table geodesic) against the FP32 product's per-ray results."""
    from parrelray_b200 import abi

    f64 = abi.FrameDesc.from_buffer_copy(frame)
    f64.precision = abi.PREC_FP64
    ref8, _, s64 = ctx.render(f64)
    mine8, _, _ = ctx.render(frame)
    d = np.abs(mine8[0].astype(np.int32) - ref8[0].astype(np.int32)).max(axis=-1)
    res = {"pixels_within_1_255_of_fp64_gpu": float(np.mean(d <= 1)), "max_abs_diff_255": int(d.max()),
           "fp64_ms": s64.kernel_ms}
    if s64.trace_ms > 0:
        # the FP64 render's tracing kernel against the measured FP64 FMA peak (same F_attempt)
        a64 = s64.attempts * F_ATTEMPT / (s64.trace_ms * 1e-3) / 1e12
        res["fp64_roofline"] = {"achieved": a64, "peak": fp64_peak, "unit": "TFLOP/s", "frac": a64 / fp64_peak,
                                "attempts": int(s64.attempts)}
    try:
        sys.path.insert(0, str(REPO / "tests"))
        from oracles import Oracle, kerr_criticality

        orc = Oracle()
    except (ImportError, FileNotFoundError):
        return res
    from parrelray_b200 import scenes

    tex = scenes.standard_textures()
    state, rgb, _ = ctx.trace_rays(frame)
    ids = np.sort(np.random.default_rng(2024).choice(frame.nrays, size=n_oracle_rays, replace=False))
    s64h, c64 = orc.trace(f64, tex, precision=1, ids=ids)
    g = state[ids]
    same = g[:, 2] == s64h[:, 2]
    band = kerr_criticality(s64h, frame.mass, frame.spin) < 0.04
    esc = same & (s64h[:, 2] == abi.RESULT_SUCCESS) & (np.linalg.norm(s64h[:, 3:6], axis=1) >= frame.rout) & ~band
    u1 = g[esc, 7:10] / np.linalg.norm(g[esc, 7:10], axis=1, keepdims=True)
    u2 = s64h[esc, 7:10] / np.linalg.norm(s64h[esc, 7:10], axis=1, keepdims=True)
    ang = np.linalg.norm(np.cross(u1, u2), axis=1)
    cd = np.abs(quantize(rgb[ids]).astype(np.int32) - quantize(c64).astype(np.int32)).max(axis=1)
    res["vs_fp64_host_oracle"] = {
        "rays": int(len(ids)), "result_agreement": float(same.mean()),
        "escaped_outside_critical_band": int(esc.sum()),
        "escape_angle_rad_p50_p99_max": [float(x) for x in np.percentile(ang, [50, 99, 100])] if esc.any() else None,
        "per_sample_colour_within_1_255": float(np.mean(cd <= 1)),
        "what": "a seeded uniform sample of the frame's rays traced by the FP64 host restatement; escape "
                "directions compared outside a +-2% band around the critical curve"}
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-trajectory", action="store_true")
    ap.add_argument("--no-uneven", action="store_true")
    ap.add_argument("--no-emission", action="store_true")
    ap.add_argument("--no-plugin", action="store_true", help="skip the Kerr plug-in header render")
    ap.add_argument("--no-refcuda", action="store_true", help="skip the reference's own CUDA build")
    ap.add_argument("--refcuda-child", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--adjoint-size", type=int, default=512, help="side of the square differentiable-render frame")
    ap.add_argument("--adam", type=int, default=200, help="iterations of the Adam fit of (a, i) (0: off)")
    ap.add_argument("--adam-lr", type=float, default=0.01)
    ap.add_argument("--adam-decay", type=float, default=0.99)
    ap.add_argument("--adam-sphere", action="store_true",
                    help="keep the workload's sphere in the fit (its edges make the loss rougher)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--plain-stride", type=int, default=1,
                    help="trajectory: render every n-th frame with the plain schedule (1: all 240)")
    ap.add_argument("--form", default="hamiltonian", choices=["hamiltonian", "contraction"],
                    help="profiling variant: the geodesic form of the timed frame (default: the product's)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"],
                    help="profiling variant: the arithmetic of the timed frame (default: the workload's FP32)")
    ap.add_argument("--launch", default=None,
                    help="block,blocks_per_sm,compaction_interval,rays_per_thread for the persistent renderer "
                         "(default: prr_autotune on the frame, outside the timed region)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.refcuda_child:
        return reference_cuda_child(args.refcuda_child, args.width, args.height)
    global RESULT_OUT
    RESULT_OUT = reserve_stdout()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch

    from parrelray_b200 import Context, LaunchConfig, abi, scenes, shard

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    ctx = Context(dev)
    tex = scenes.standard_textures()
    ctx.upload_textures(tex)
    frames = orbit_frames(ws, args.width, args.height)
    variant = {}
    if args.precision == "fp64":  # profiling variants, named in the output's config
        for f in frames:
            f.precision = abi.PREC_FP64
        variant["precision"] = "fp64"
    ham_mask = abi.HAM_FP32 | abi.HAM_FP64
    if args.form == "contraction":
        ham_mask = 0
        ctx.set_option(abi.OPT_HAMILTONIAN, ham_mask)
        variant["form"] = "contraction"
    frame = frames[rank]  # this rank's share when every rank draws one frame (weak scaling)
    npx = frame.width * frame.height
    t_tune = time.perf_counter()
    if args.launch:
        b, bp, ci, rpt = (int(v) for v in args.launch.split(","))
        ctx.set_schedule(abi.SCHED_PERSISTENT, LaunchConfig(b, bp, ci, rpt))
        tuned_on = "given on the command line"
    else:
        # the launch shape does not change the arithmetic of a ray; it is tuned on the frame itself
        # (on a half-size copy the tail of the persistent launch weighs more and favours fewer threads)
        ctx.autotune(frame)
        tuned_on = "prr_autotune on the frame itself, outside the timed region"
    t_tune = time.perf_counter() - t_tune
    out8 = torch.empty(npx * 3, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    stream = torch.cuda.current_stream()
    ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def render_claimed(fs):
        """This rank's renderer for shard.render_sharded: device outputs, CUDA-event time."""
        ev_a.record(stream)
        for f in fs:
            ctx.render_device(f, out8.data_ptr(), stream=stream.cuda_stream)
        ev_b.record(stream)
        ev_b.synchronize()
        return [None] * len(fs), ev_a.elapsed_time(ev_b)

    def step():
        flush.zero_()
        if ws > 1:
            # the step's frames are pulled from a shared counter (shard.py), each rank rendering what it claims
            shard.render_sharded(frames, render_claimed, gather_to=None)
        else:
            ctx.render_device(frame, out8.data_ptr(), stream=stream.cuda_stream)

    # warm-up (also the stats of one frame: attempts for the roofline)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _, _, st = ctx.render(frame)

    sampler = ClockSampler(dev)
    sampler.start()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    if ws > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    rays = frame.nrays
    value = ws * rays / (ms * 1e-3) / 1e6

    # ---- e2e through the public API with host buffers ----
    host8 = torch.empty(npx * 3, dtype=torch.uint8, pin_memory=True).numpy()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.render(frame, out8=host8)
    barrier()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    if ws > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = {"value": ws * rays / (e2e_ms * 1e-3) / 1e6, "unit": "Mrays/s",
           "h2d_bytes_per_step": int(abi.C.sizeof(abi.FrameDesc)), "d2h_bytes_per_step": int(npx * 3)}

    extra = {}
    if rank == 0:
        fp32_peak, fp64_peak = ctx.measure_peak()
        achieved = st.attempts * F_ATTEMPT / (st.trace_ms * 1e-3) / 1e12
        kname = pair_kernel_name(ctx.launch_config())
        ncu_flop = NCU_FLOP_PER_ATTEMPT["k_ham" if kname.startswith("k_ham") else "k_pair"]
        counted = st.attempts * ncu_flop / (st.trace_ms * 1e-3) / 1e12
        roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp32_peak, "traffic": TRAFFIC_PER_LAUNCH,
                    "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one launch of the tracing "
                                      "kernel on the 960x540 copy of this frame (ncu): the textures; they do not "
                                      "grow with the frame, and the outputs stay in L2",
                    "kernel": pair_kernel_name(ctx.launch_config()), "kernel_ms": st.trace_ms,
                    "flop_per_attempt": F_ATTEMPT, "attempts": st.attempts,
                    "frac_basis": "algorithmic: attempts x F_attempt (the work of one RKF45 attempt of the (x, u) "
                                  "system in the Kerr-Schild contraction form, FMA = 2; ncu counts 1,459 executed "
                                  "for it) / kernel time",
                    "ncu_counted": {"achieved": counted, "frac": counted / fp32_peak,
                                    "flop_per_attempt": ncu_flop, "rule": NCU_FLOP_RULE,
                                    "note": "the FP32 work the kernel executes; the Hamiltonian form does one "
                                            "attempt in fewer operations than F_attempt counts"},
                    "peak_source": "measured on this GPU: FMA-chain kernel (prr_measure_peak), burst",
                    "fp64_peak_tflops": fp64_peak}
        extra["roofline"] = roofline
        extra["stats"] = {k: v for k, v in st.as_dict().items()}
        if not args.no_plain and ws == 1:
            def timed_device(n=1):
                ctx.render(frame)  # warm-up of this configuration
                ev0.record(stream)
                for _ in range(n):
                    ctx.render_device(frame, out8.data_ptr(), stream=stream.cuda_stream)
                ev1.record(stream)
                torch.cuda.synchronize()
                return ev0.elapsed_time(ev1) / n

            ctx.set_schedule(abi.SCHED_PLAIN)
            plain_ms = timed_device()                      # reference structure + Christoffel table
            ctx.set_option(abi.OPT_GEOD_TABLE, 0)
            plain_contraction_ms = timed_device()          # reference structure + register contraction
            ctx.set_schedule(abi.SCHED_PERSISTENT)
            ctx.set_option(abi.OPT_GEOD_TABLE, 1)
            table_ms = timed_device()                      # persistent scheduler + Christoffel table
            ctx.set_option(abi.OPT_GEOD_TABLE, -1)
            ctx.set_option(abi.OPT_HAMILTONIAN, abi.HAM_FP64)
            contraction_ms = timed_device()                # persistent scheduler + contraction, (x, u) state
            ctx.set_option(abi.OPT_HAMILTONIAN, ham_mask)
            extra["plain"] = {"value": rays / (plain_ms * 1e-3) / 1e6, "ms_per_step": plain_ms,
                              "speedup": plain_ms / ms,
                              "speedup_scheduler_only": plain_contraction_ms / contraction_ms,
                              "speedup_scheduler_only_table": plain_ms / table_ms,
                              "speedup_geodesic_form_only": plain_ms / plain_contraction_ms,
                              "speedup_hamiltonian_form": contraction_ms / ms,
                              "what": "one ray per thread, 64-row layers, AoS rays in HBM, textbook stages, "
                                      "Christoffel-table geodesic; speedup = all changes; scheduler_only = the "
                                      "persistent compaction scheduler with the geodesic form held fixed (contraction, "
                                      "or table); geodesic_form_only = contraction against table on the plain "
                                      "schedule; hamiltonian_form = the (x, p) state against the (x, u) contraction "
                                      "on the persistent schedule",
                              "breakdown_ms": {"plain_table": plain_ms, "plain_contraction": plain_contraction_ms,
                                               "persistent_table": table_ms, "persistent_contraction": contraction_ms,
                                               "persistent_hamiltonian": ms}}
        if not args.no_adjoint and ws == 1:
            # discrete adjoint of the 512x512 differentiable-render workload: one gradient of an L2 image loss
            n = args.adjoint_size
            _, tgt, _ = ctx.render(scenes.kerr_512_adjoint(spin=0.7, precision=abi.PREC_FP32, size=n), want_float=True)
            res = {"unit": "ms", "workload": f"kerr a=0.3 i=45 r=20, {n}x{n}, 1 sphere, bilinear sky, tol 1e-6; "
                                             "d(L2 to the a=0.7 render)/d(a, M, i, r, phase), checkpoints every 64 "
                                             "accepted steps"}
            for prec, key in ((abi.PREC_FP32, "fp32_forward"), (abi.PREC_FP64, "fp64_forward")):
                start = scenes.kerr_512_adjoint(spin=0.3, incl_deg=45.0, precision=prec, size=n)
                _, cur, _ = ctx.render(start, want_float=True)
                dl = 2.0 * (cur[0] - tgt[0])
                for _ in range(2):  # the first call sizes the checkpoint buffer
                    g, ast = ctx.adjoint(start, dl, 0)
                res[key] = {"ms": ast.kernel_ms, "forward_render_ms": ast.trace_ms, "grad": g.tolist(),
                            "accepted_steps": ast.accepted}
            # the workload's form (FP32 forward steps, FP64 adjoint and reduction) is the headline number
            res["ms"] = res["fp32_forward"]["ms"]
            extra["adjoint"] = res
        if args.adam > 0 and ws == 1:
            extra["adam_fit"] = bench_adam_fit(ctx, args.adam, args.adjoint_size, args.adam_lr, args.adam_decay,
                                               args.adam_sphere)
        if not args.no_trajectory and ws == 1:
            extra["trajectory"] = bench_trajectory(ctx, torch, stream, plain_stride=args.plain_stride)
        if not args.no_uneven and ws == 1:
            extra["uneven"] = bench_uneven(ctx, torch, stream, tex)
        if not args.no_emission and ws == 1:
            extra["emission"] = bench_emission(ctx, torch, stream)
        ctx.upload_textures(tex)
        if not args.no_plugin and ws == 1:
            extra["plugin_kerr_header"] = bench_plugin_kerr(ctx, torch, stream, frame)
        if not args.no_accuracy and ws == 1:
            extra["accuracy"] = bench_accuracy(ctx, frame, fp64_peak)
        if not args.no_cpu and ws == 1:
            # the cpu_baseline leg: the CPU restatement and the reference's host build, on this host's cores
            sys.path.insert(0, str(REPO / "tests"))
            try:
                from oracles import Oracle

                orc = Oracle()
            except (ImportError, FileNotFoundError):
                orc = None
            nthreads = os.cpu_count() or 1
            if orc is not None:
                f64 = abi.FrameDesc.from_buffer_copy(frame)
                f64.precision = abi.PREC_FP64
                ids = calibrated_ray_sample(orc, f64, tex, args.cpu_seconds, nthreads)
                r = oracle_fp64_sample(orc, f64, tex, ids, nthreads)
                extra["cpu_baseline"] = {
                    "value": r["mrays_s"], "unit": "Mrays/s", "cores": nthreads, "kind": "port",
                    "sample": f"{r['rays']} rays drawn uniformly (seed 2024) from the frame, FP64 PHYSICAL "
                              f"restatement (oracle/prr_oracle.cpp) at tolerance 1e-6, {r['seconds']:.1f} s"}
                ctxr = cpu_reference_sample(frame, tex, 4.0, nthreads, eps=1e-3)
                if ctxr:
                    extra["cpu_baseline"]["reference_solver_eps_1e-3"] = ctxr
            extra.setdefault("cpu_baseline", {})["single_frame_workload"] = single_frame_workload(ctx, nthreads)
            ctx.upload_textures(tex)
        if not args.no_refcuda and ws == 1:
            rc = bench_reference_cuda(args.width, args.height)
            if "eps_1e-3_frame" in rc:
                # the same frame, algorithm and tolerance through this library's REFERENCE mode
                # (one thread per ray, fused placement/init/trace/colour; the geodesic by the
                # Kerr-Schild contraction where the reference's plug-in header uses a table)
                rf = scenes.kerr_1080p_ssaa4(args.width, args.height, mode=abi.MODE_REFERENCE, eps=1e-3,
                                             horizon_eps=0.001)
                ctx.render(rf)
                _, _, rst = ctx.render(rf)
                rc["eps_1e-3_frame"]["this_library_reference_mode_s"] = rst.kernel_ms * 1e-3
                rc["eps_1e-3_frame"]["speedup_of_this_library"] = rc["eps_1e-3_frame"]["seconds"] / (rst.kernel_ms * 1e-3)
            extra["reference_cuda"] = rc
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural textures)",
            "config": dict(workload_config(args.width, args.height), **({"variant": variant} if variant else {})),
            "launch": {"schedule": "persistent" + (", frames pulled from a shared counter" if ws > 1 else ""),
                       "shape": {k: getattr(ctx.launch_config(), k) for k, _ in LaunchConfig._fields_},
                       "source": tuned_on, "autotune_s": round(t_tune, 2)},
            "e2e": e2e, "clocks": clocks, "gpu_launches": int(st.kernel_launches) * args.steps,
        }
        line.update(extra)
        emit(line)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
