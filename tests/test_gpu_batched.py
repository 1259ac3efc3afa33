"""Recorded batches (prr_graph_*) and split precision over uneven requests.

* A camera trajectory (the 240-frame Kerr a = 0.9 orbit-descent workload at
  reduced frame count and size) recorded into one CUDA graph replays to the
  same bytes as prr_render of the same batch and as per-frame renders, on
  every replay; prr_graph_set_frames swaps in new frames without
  re-recording; the tuned launch shape is the one recorded.
* Uneven requests (the 64-request workload: log-uniform resolutions, spin,
  distance and inclination drawn from a fixed seed; tolerance 1e-7) in SPLIT
  precision: each request within 1/255 of the all-FP64 GPU render on
  >= 99.9% of its pixels overall, never worse than the FP32 render, and the
  graph replays the split render bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import pixel_rule, quantize
from parrelray_b200 import Graph, abi, scenes

pytestmark = pytest.mark.gpu


def _torch_out(nbytes, dtype):
    import torch

    return torch.zeros(nbytes, dtype=dtype, device="cuda")


def split_images(flat, frames):
    out, off = [], 0
    for f in frames:
        n = f.width * f.height * 3
        out.append(flat[off:off + n].reshape(f.height, f.width, 3))
        off += n
    return out


@pytest.fixture(scope="module")
def traj(small_textures):
    return scenes.trajectory_240(n=24, width=96, height=54)


def test_graph_replays_equal_batched_and_per_frame_renders(gpu, small_textures, traj):
    import torch

    gpu.upload_textures(small_textures)
    npx = sum(f.width * f.height for f in traj)
    ref, _, st_ref = gpu.render(traj)
    per_frame = [gpu.render(f)[0][0] for f in traj]
    for a, b in zip(ref, per_frame):
        assert np.array_equal(a, b)
    out8 = _torch_out(npx * 3, torch.uint8)
    outf = _torch_out(npx * 3, torch.float32)
    with Graph(gpu, traj, out8.data_ptr(), outf.data_ptr()) as g:
        for rep in range(2):
            out8.zero_()
            g.launch(torch.cuda.current_stream().cuda_stream)
            st = g.stats()
            got = split_images(out8.cpu().numpy(), traj)
            for k, (a, b) in enumerate(zip(got, ref)):
                assert np.array_equal(a, b), f"replay {rep} frame {k}"
            assert st.rays == st_ref.rays and st.attempts == st_ref.attempts and st.accepted == st_ref.accepted
            assert st.kernel_launches == 1  # one persistent launch for the whole trajectory
        fl = outf.cpu().numpy()
        assert np.array_equal(quantize(fl.reshape(-1, 3)), out8.cpu().numpy().reshape(-1, 3))


def test_graph_set_frames_without_rerecording(gpu, small_textures, traj):
    import torch

    gpu.upload_textures(small_textures)
    later = scenes.trajectory_240(n=24, width=96, height=54, spin=0.5)
    ref, _, _ = gpu.render(later)
    npx = sum(f.width * f.height for f in traj)
    out8 = _torch_out(npx * 3, torch.uint8)
    with Graph(gpu, traj, out8.data_ptr()) as g:
        g.launch()
        g.stats()
        g.set_frames(later)
        g.launch()
        g.stats()
        got = split_images(out8.cpu().numpy(), later)
        assert all(np.array_equal(a, b) for a, b in zip(got, ref))
        bigger = scenes.trajectory_240(n=24, width=97, height=54)
        with pytest.raises(abi.PrrError) as e:
            g.set_frames(bigger)
        assert e.value.status == abi.ERR_INVALID
        with pytest.raises(abi.PrrError):
            g.set_frames(later[:5])


def test_graph_records_the_tuned_launch_shape(gpu, small_textures, traj):
    import torch

    gpu.upload_textures(small_textures)
    saved = gpu.launch_config()
    try:
        best = gpu.autotune(traj[0])
        assert best.block_size in (64, 128, 256) and best.compaction_interval >= 1
        out8 = _torch_out(sum(f.width * f.height for f in traj) * 3, torch.uint8)
        ref, _, _ = gpu.render(traj)
        with Graph(gpu, traj, out8.data_ptr()) as g:
            rec = g.launch_config()
            assert (rec.block_size, rec.compaction_interval) == (best.block_size, best.compaction_interval)
            assert rec.blocks_per_sm >= 1
            g.launch()
            g.stats()
            got = split_images(out8.cpu().numpy(), traj)
            if rec.rays_per_thread == 1:  # the block shape and refill interval do not change a ray's arithmetic
                assert all(np.array_equal(a, b) for a, b in zip(got, ref))
            else:  # two rays per thread round a few operations differently
                assert all(pixel_rule(a, b) >= 0.999 for a, b in zip(got, ref))
    finally:
        gpu.set_schedule(abi.SCHED_PERSISTENT, saved)


def test_graph_rejects_reference_mode_and_missing_outputs(gpu, small_textures):
    gpu.upload_textures(small_textures)
    d = scenes.schwarzschild_320(mode=abi.MODE_REFERENCE, horizon_eps=0.001)
    h = C.c_void_p()
    st = abi.load().prr_graph_create(gpu.h, C.byref(d), 1, C.c_void_p(1 << 20), None, C.byref(h))
    assert st == abi.ERR_UNSUPPORTED and not h.value
    d = scenes.schwarzschild_320()
    st = abi.load().prr_graph_create(gpu.h, C.byref(d), 1, None, None, C.byref(h))
    assert st == abi.ERR_INVALID and not h.value


@pytest.fixture(scope="module")
def uneven(gpu, small_textures):
    """64 uneven requests, each capped at 3072 pixels to keep the FP64 render short."""
    gpu.upload_textures(small_textures)
    reqs = {p: scenes.uneven_64(max_pixels=3072, precision=p) for p in (abi.PREC_FP32, abi.PREC_FP64, abi.PREC_SPLIT)}
    out = {}
    for p, fr in reqs.items():
        imgs, _, st = gpu.render(fr)
        out[p] = (imgs, st)
    return reqs, out


def test_split_precision_per_request_error(uneven):
    reqs, out = uneven
    ref = out[abi.PREC_FP64][0]
    split, st_split = out[abi.PREC_SPLIT]
    fp32 = out[abi.PREC_FP32][0]
    assert st_split.n_fp64 > 0, "no ray was routed to the FP64 pass"
    assert st_split.n_fp64 < 0.25 * st_split.rays
    per_req = np.array([pixel_rule(a, b) for a, b in zip(split, ref)])
    bad_split = sum(int(np.sum(np.abs(a.astype(int) - b.astype(int)).max(-1) > 1)) for a, b in zip(split, ref))
    bad_fp32 = sum(int(np.sum(np.abs(a.astype(int) - b.astype(int)).max(-1) > 1)) for a, b in zip(fp32, ref))
    total = sum(a.shape[0] * a.shape[1] for a in ref)
    assert bad_split / total <= 1e-3, (bad_split, total)
    assert per_req.min() >= 0.99, per_req.min()
    assert bad_split <= bad_fp32, (bad_split, bad_fp32)


def test_split_requests_batched_equal_single(gpu, small_textures, uneven):
    reqs, out = uneven
    gpu.upload_textures(small_textures)
    fr = reqs[abi.PREC_SPLIT]
    for k in (0, 17, 63):
        single = gpu.render(fr[k])[0][0]
        assert np.array_equal(single, out[abi.PREC_SPLIT][0][k]), k


def test_split_graph_equals_render(gpu, small_textures, uneven):
    import torch

    reqs, out = uneven
    gpu.upload_textures(small_textures)
    fr = reqs[abi.PREC_SPLIT]
    out8 = _torch_out(sum(f.width * f.height for f in fr) * 3, torch.uint8)
    with Graph(gpu, fr, out8.data_ptr()) as g:
        g.launch()
        st = g.stats()
        got = split_images(out8.cpu().numpy(), fr)
    assert all(np.array_equal(a, b) for a, b in zip(got, out[abi.PREC_SPLIT][0]))
    assert st.n_fp64 == out[abi.PREC_SPLIT][1].n_fp64


def test_split_matches_fp64_oracle_on_small_requests(gpu, oracle, small_textures):
    """Four requests of the uneven workload at 40x24 against the FP64 host oracle."""
    gpu.upload_textures(small_textures)
    fr = [f for f in scenes.uneven_64(max_pixels=960, precision=abi.PREC_SPLIT)][:4]
    imgs, _, _ = gpu.render(fr)
    for f, img in zip(fr, imgs):
        f64 = abi.FrameDesc.from_buffer_copy(f)
        f64.precision = abi.PREC_FP64
        _, _, ref = oracle.render(f64, small_textures, precision=1)
        assert pixel_rule(img, quantize(ref)) >= 0.99
