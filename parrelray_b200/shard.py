"""Multi-GPU sharding of a batch of frames: one process per GPU, no
collective on the data path.

Every frame (and every ray of it) is independent, so a trajectory or a set
of render requests is split over the ranks and each rank renders its share
with one batched call on its own GPU.  The only communication is the final
gather of the 8-bit images to one rank (or none, when every rank writes its
own frames) and the max-over-ranks device time.  The reference renders
frames one after another on one GPU (prr.cpp:382-386).

`assign` balances ranks by ray count (frames of a trajectory differ in
cost only through their content, so rays are the known weight), keeping each
rank's frames in trajectory order.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def assign(weights: Sequence[int], world: int) -> list[list[int]]:
    """Frame indices per rank: greedy longest-processing-time over
    `weights` (rays per frame), then each rank's list sorted.  Every frame
    goes to exactly one rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-int(weights[i]), i))
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += int(weights[i])
    return [sorted(x) for x in out]


def render_sharded(frames: Sequence, render: Callable[[list], tuple[list[np.ndarray], float]], group=None,
                   gather_to: int | None = 0):
    """Renders `frames` across the ranks of the default process group.

    render(list_of_frames) -> (list of (h, w, 3) uint8 images, device ms) is
    this rank's renderer (e.g. one prr_render call on its GPU).  Returns
    (images or None, max_ms): rank `gather_to` receives every frame's image
    in the original order (None on the other ranks; gather_to=None keeps each
    rank's own frames, in its assignment order); max_ms is the slowest
    rank's device time, the number a multi-GPU throughput is quoted on."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    weights = [int(f.width) * int(f.height) * int(f.samples) for f in frames]
    plan = assign(weights, world)
    mine = plan[rank]
    imgs, ms = render([frames[i] for i in mine]) if mine else ([], 0.0)
    t = torch.tensor([float(ms)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    max_ms = float(t.item())
    if gather_to is None:
        return list(zip(mine, imgs)), max_ms
    payload = [(i, np.ascontiguousarray(im)) for i, im in zip(mine, imgs)]
    gathered = [None] * world if rank == gather_to else None
    dist.gather_object(payload, gathered, dst=gather_to, group=group)
    if rank != gather_to:
        return None, max_ms
    out: list = [None] * len(frames)
    for part in gathered:
        for i, im in part:
            out[i] = im
    assert all(o is not None for o in out), "a frame was not rendered by any rank"
    return out, max_ms
