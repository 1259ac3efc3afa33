"""Multi-GPU sharding host logic on CPU: two `gloo` ranks (world_size 2),
each standing in for one GPU process.  The per-rank renderer here is the
FP64 CPU oracle on tiny frames (the checker), so the test exercises the
partition, the max-over-ranks time and the ordered gather to rank 0 without
a GPU.  The GPU path runs the same code with a prr_render call per rank."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from parrelray_b200 import shard

HERE = Path(__file__).resolve().parent


def test_assign_balances_and_covers():
    w = [5, 1, 1, 1, 9, 3, 3, 2]
    for world in (1, 2, 3, 8, 10):
        plan = shard.assign(w, world)
        flat = sorted(i for p in plan for i in p)
        assert flat == list(range(len(w)))
        assert all(p == sorted(p) for p in plan)
        loads = [sum(w[i] for i in p) for p in plan]
        assert max(loads) - min(loads) <= max(w)
    with pytest.raises(ValueError):
        shard.assign(w, 0)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, str(HERE))
    sys.path.insert(0, str(HERE.parent))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from oracles import Oracle
    from parrelray_b200 import abi, scenes
    from parrelray_b200 import shard as sh

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    tex = {scenes.SKY_ID: scenes.make_texture(1, 1234, 64, 32), scenes.SPHERE_ID0: scenes.make_texture(0, 100, 32, 16)}
    frames = scenes.trajectory_240(n=5, width=12, height=8, precision=abi.PREC_FP64)
    orc = Oracle()

    def render(fs):
        imgs = []
        for f in fs:
            _, _, img = orc.render(f, tex, precision=1)
            imgs.append(np.floor(np.clip(img, 0, 1) * 255 + 0.5).astype(np.uint8))
        return imgs, 10.0 * (rank + 1)  # distinct per-rank "device time"

    imgs, ms = sh.render_sharded(frames, render)
    own, _ = sh.render_sharded(frames, render, gather_to=None)
    if rank == 0:
        np.savez(Path(out_dir) / "gathered.npz", *imgs, ms=ms)
    np.save(Path(out_dir) / f"own{rank}.npy", np.array([i for i, _ in own]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.slow
def test_two_gloo_ranks_render_and_gather(built, tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    z = np.load(tmp_path / "gathered.npz")
    assert float(z["ms"]) == 20.0  # max over ranks
    got = [z[f"arr_{i}"] for i in range(5)]
    # each frame once, in order: compare with a single-process render
    from oracles import Oracle
    from parrelray_b200 import abi, scenes

    tex = {scenes.SKY_ID: scenes.make_texture(1, 1234, 64, 32), scenes.SPHERE_ID0: scenes.make_texture(0, 100, 32, 16)}
    orc = Oracle()
    for f, g in zip(scenes.trajectory_240(n=5, width=12, height=8, precision=abi.PREC_FP64), got):
        _, _, img = orc.render(f, tex, precision=1)
        assert np.array_equal(np.floor(np.clip(img, 0, 1) * 255 + 0.5).astype(np.uint8), g)
    own = sorted(np.load(tmp_path / "own0.npy").tolist() + np.load(tmp_path / "own1.npy").tolist())
    assert own == list(range(5))
