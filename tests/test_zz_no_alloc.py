"""prr_render_noalloc, the entry point for callers that cannot allocate
device memory while rendering (an application that reserves its whole device
budget up front and hands out pieces of it itself, or a real-time loop that
must not pay cudaMalloc's implicit synchronisation).  The caller owns the
textures and outputs; the library's only scratch is a fixed static device
array.

Checked through the C ABI against the context entry point prr_render on the
same frames, on two calls in a row (the second call reuses the scratch the
first left behind).  This file is collected last so that a run stopping at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from parrelray_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def frames_pair(precision=abi.PREC_FP32):
    sph = [(*scenes.orbit_point(orb, ph), rad, scenes.SPHERE_ID0 + k)
           for k, (rad, orb, ph) in enumerate(scenes.KERR_1080P_SPHERES)]
    a = scenes.make_frame(64, 36, r=25.0, incl_deg=80.0, fov_deg=50.0, metric=abi.METRIC_KERR, spin=0.95, samples=4,
                          fxaa=True, spheres=sph, precision=precision)
    b = scenes.make_frame(48, 30, r=20.0, incl_deg=60.0, fov_deg=60.0, metric=abi.METRIC_SCHWARZSCHILD, samples=1,
                          fxaa=False, spheres=sph[:1], precision=precision)
    return [a, b]


FRAME_SETS = {
    # the FP32 renderer on a Kerr frame with SSAA + FXAA and a Schwarzschild frame without
    "fp32": lambda: frames_pair(abi.PREC_FP32),
    # the same frames through the FP64 renderer
    "fp64": lambda: frames_pair(abi.PREC_FP64),
    # plasma emission from a thick disk (the FP32 renderer's emission instantiation)
    "emission": lambda: [scenes.eht_disk(48, samples=4)],
}


def device_textures(textures):
    import torch

    keep = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in textures.items()}
    ptrs = (C.c_void_p * abi.PRR_MAX_TEXTURES)()
    w = (C.c_int32 * abi.PRR_MAX_TEXTURES)()
    h = (C.c_int32 * abi.PRR_MAX_TEXTURES)()
    for k, t in keep.items():
        ptrs[k] = t.data_ptr()
        h[k], w[k] = t.shape[0], t.shape[1]
    return keep, ptrs, w, h


@pytest.mark.parametrize("kind", sorted(FRAME_SETS))
def test_noalloc_matches_context_render_on_two_calls(gpu, small_textures, kind):
    import torch

    from parrelray_b200 import LaunchConfig

    lib = abi.load()
    frames = FRAME_SETS[kind]()
    gpu.upload_textures(small_textures)
    # the context renders with the launch shape the entry point uses (64-thread CTAs at their
    # occupancy limit, a refill every 64 attempts), so both run the same kernel instantiation
    saved = gpu.launch_config()
    gpu.set_schedule(abi.SCHED_PERSISTENT, LaunchConfig(64, 0, 64, 1))
    try:
        ref8, reff, _ = gpu.render(frames, want_float=True)
    finally:
        gpu.set_schedule(abi.SCHED_PERSISTENT, saved)
    keep, ptrs, w, h = device_textures(small_textures)
    npx = sum(f.width * f.height for f in frames)
    out8 = torch.empty(npx * 3, dtype=torch.uint8, device="cuda")
    outf = torch.empty(npx * 3, dtype=torch.float32, device="cuda")
    arr = (abi.FrameDesc * len(frames))(*frames)
    stream = torch.cuda.current_stream().cuda_stream
    err = C.create_string_buffer(512)
    for call in range(2):
        out8.fill_(7)
        outf.fill_(-1.0)
        st = lib.prr_render_noalloc(arr, len(frames), ptrs, w, h, out8.data_ptr(), outf.data_ptr(), stream, err, 512)
        assert st == abi.OK, err.value.decode()
        torch.cuda.synchronize()
        got8 = out8.cpu().numpy()
        gotf = outf.cpu().numpy()
        off = 0
        for k, f in enumerate(frames):
            n = f.width * f.height * 3
            img8 = got8[off:off + n].reshape(f.height, f.width, 3)
            # same kernels on the same frames: identical bytes
            assert np.array_equal(img8, ref8[k]), f"{kind}: call {call}, frame {k}"
            if not f.fxaa:  # with FXAA, d_rgbf holds the pre-FXAA combined image
                assert np.array_equal(gotf[off:off + n].reshape(f.height, f.width, 3), reff[k])
            off += n


def test_noalloc_rejects_more_frames_than_its_scratch_holds(gpu, small_textures):
    import torch

    lib = abi.load()
    f = frames_pair()[1]
    n = 65  # PRR_NOALLOC_MAX_FRAMES + 1
    arr = (abi.FrameDesc * n)(*([f] * n))
    keep, ptrs, w, h = device_textures(small_textures)
    out8 = torch.empty(n * f.width * f.height * 3, dtype=torch.uint8, device="cuda")
    err = C.create_string_buffer(512)
    st = lib.prr_render_noalloc(arr, n, ptrs, w, h, out8.data_ptr(), None, None, err, 512)
    assert st == abi.ERR_INVALID
    assert b"at most 64" in err.value
