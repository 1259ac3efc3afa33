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


def test_guided_claims_cover_each_item_once():
    for n, world in ((0, 2), (1, 2), (7, 1), (40, 2), (240, 8), (5, 16)):
        box = [0]

        def add(k):
            box[0] += k
            return box[0]

        # interleave two claimants on one counter as ranks would
        claims = list(shard.guided_claims(n, world, add))
        got = sorted(i for b, e in claims for i in range(b, e))
        assert got == list(range(n))
        sizes = [e - b for b, e in claims]
        assert all(s >= 1 for s in sizes)
        assert sizes == sorted(sizes, reverse=True) or n == 0  # claims shrink as the work runs out


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

    _, ms = sh.render_sharded(frames, render, schedule="static")  # one call per rank: its time is known
    imgs, _ = sh.render_sharded(frames, render)  # frames pulled from the shared counter
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


# Per-frame cost of the uneven batch: every even frame costs 5x an odd one, while all frames have
# the same number of rays, so a split by rays puts all the expensive frames on one rank.
def _uneven_cost_ms(k: int) -> float:
    return 20.0 if k % 2 == 0 else 4.0


def _uneven_worker(rank, world, port, out_dir, schedule):
    sys.path.insert(0, str(HERE.parent))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import time

    import torch.distributed as dist

    from parrelray_b200 import shard as sh

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))

    class Frame:  # equal rays everywhere
        width, height, samples = 64, 36, 1

        def __init__(self, k):
            self.k = k

    frames = [Frame(k) for k in range(40)]

    def render(fs):
        t = 0.0
        for f in fs:
            c = _uneven_cost_ms(f.k)
            time.sleep(c * 1e-3)  # stands in for the GPU's work on this frame
            t += c
        return [f.k for f in fs], t

    dist.barrier()  # both ranks start claiming together, as GPU ranks do after their set-up
    own, _ = sh.render_sharded(frames, render, gather_to=None, schedule=schedule)
    np.save(Path(out_dir) / f"{schedule}{rank}.npy", np.array([i for i, _ in own], dtype=np.int64))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.slow
def test_pulled_frames_balance_uneven_costs(tmp_path):
    """Two gloo ranks render a batch whose frames have equal rays but costs that differ 5x: pulling
    frames from the shared counter keeps the ranks' work within 1.2 of each other, where the
    static split by rays leaves them 5x apart."""
    world = 2
    loads = {}
    for schedule in ("pull", "static"):
        mp.start_processes(_uneven_worker, args=(world, _free_port(), str(tmp_path), schedule), nprocs=world,
                           join=True, start_method="spawn")
        parts = [np.load(tmp_path / f"{schedule}{r}.npy").tolist() for r in range(world)]
        assert sorted(parts[0] + parts[1]) == list(range(40))
        loads[schedule] = [sum(_uneven_cost_ms(k) for k in p) for p in parts]
    lp, ls = loads["pull"], loads["static"]
    assert max(lp) / min(lp) <= 1.2, lp
    assert max(ls) / min(ls) >= 4.0, ls
