"""Multi-GPU sharding of a batch of frames: one process per GPU, no
collective on the data path.

Every frame (and every ray of it) is independent, so a trajectory or a set
of render requests is split over the ranks and each rank renders its share
on its own GPU.  The only communication is a shared work counter in the
process group's store (a few bytes per claim), the final gather of the 8-bit
images to one rank (or none, when every rank keeps its own frames) and the
max-over-ranks device time.  The reference renders frames one after another
on one GPU (prr.cpp:382-386).

Frames of one batch can differ in cost by orders of magnitude (ray lifetimes
run from ~50 to ~10,000 steps, and a close camera or a high spin costs more
per ray), so pixel or ray counts are a poor estimate of a frame's cost.  The
default schedule therefore does not estimate: ranks pull frames from the
shared counter (guided self-scheduling: a claim takes about a 1/(2 world) share
of the frames still unclaimed, at least one), so a rank that drew cheap frames
simply claims more, and ranks finish within about one frame of each other.
`assign` is the static alternative (longest-processing-time greedy over
given weights), used when the weights are known.
"""
from __future__ import annotations

import itertools
from typing import Callable, Sequence

import numpy as np

_CALLS = itertools.count()


def assign(weights: Sequence[float], world: int) -> list[list[int]]:
    """Frame indices per rank: greedy longest-processing-time over
    `weights` (the expected cost of each frame), then each rank's list
    sorted.  Every frame goes to exactly one rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(weights[i])
    return [sorted(x) for x in out]


def guided_claims(n: int, world: int, counter):
    """Yields [begin, end) ranges of `n` work items claimed through
    `counter(k)`, an atomic fetch-and-add that returns the counter's value
    after adding k (counter(0) reads it).  A claim is made only when the
    previous range has been consumed (the generator is lazy), and asks for
    ceil(remaining / (2 world)) items, remaining read just before, at least
    1; the ranges of all ranks are disjoint and cover [0, n)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    while True:
        seen = int(counter(0))
        if seen >= n:
            return
        k = max(1, -(-(n - seen) // (2 * world)))
        end = int(counter(k))
        begin = end - k
        if begin >= n:
            return
        yield begin, min(end, n)
        if end >= n:
            return


def _store():
    """The default process group's key-value store (every rank reaches it)."""
    import torch.distributed as dist

    return dist.distributed_c10d._get_default_store()


def render_sharded(frames: Sequence, render: Callable[[list], tuple[list, float]], group=None,
                   gather_to: int | None = 0, schedule: str = "pull", weights: Sequence[float] | None = None):
    """Renders `frames` across the ranks of the process group.

    render(list_of_frames) -> (list of per-frame results, device ms) is this
    rank's renderer (e.g. one prr_render call on its GPU; a result is
    typically an (h, w, 3) uint8 image).  schedule "pull" claims frames from
    the shared counter (see the module docstring); "static" splits them once
    by `weights` (default: rays per frame).  Every rank must make the same
    calls in the same order.  Returns (results or None, max_ms): rank
    `gather_to` receives every frame's result in the original order (None on
    the other ranks; gather_to=None keeps each rank's own frames as (index,
    result) pairs); max_ms is the slowest rank's summed device time, the
    number a multi-GPU throughput is quoted on."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine: list[tuple[int, object]] = []
    ms = 0.0
    if schedule == "pull":
        key = f"prr_shard_{next(_CALLS)}"
        store = _store()
        for b, e in guided_claims(len(frames), world, lambda k: store.add(key, k)):
            res, t = render([frames[i] for i in range(b, e)])
            mine.extend(zip(range(b, e), res))
            ms += float(t)
    elif schedule == "static":
        w = weights if weights is not None else [int(f.width) * int(f.height) * int(f.samples) for f in frames]
        idx = assign(w, world)[rank]
        if idx:
            res, t = render([frames[i] for i in idx])
            mine = list(zip(idx, res))
            ms = float(t)
    else:
        raise ValueError("schedule must be 'pull' or 'static'")
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"  # NCCL reduces device tensors only
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    max_ms = float(t.item())
    if gather_to is None:
        return mine, max_ms
    payload = [(i, np.ascontiguousarray(r) if isinstance(r, np.ndarray) else r) for i, r in mine]
    gathered = [None] * world if rank == gather_to else None
    dist.gather_object(payload, gathered, dst=gather_to, group=group)
    if rank != gather_to:
        return None, max_ms
    out: list = [None] * len(frames)
    for part in gathered:
        for i, r in part:
            out[i] = r
    assert all(o is not None for o in out), "a frame was not rendered by any rank"
    return out, max_ms
