"""The multi-rank path on CPU: gloo, world size 2. Frame sharding covers every
frame once with good balance, and the gather returns every rank's frames to
rank 0 in frame order (the N>1 bench and batched renders use the same
helpers)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rtwca_b200 import configs, shard


def test_assign_frames_covers_and_balances():
    _, cams, _, meta = configs.batched_frames(96, seed=0)
    costs = [shard.frame_cost(c.x_pix, c.y_pix, c.tolerance) for c in cams]
    for world in (1, 2, 4, 8):
        a = shard.assign_frames(costs, world)
        flat = sorted(i for part in a for i in part)
        assert flat == list(range(96))
        assert shard.balance(costs, a) < 1.05


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, result_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        _, cams, _, _ = configs.batched_frames(12, seed=0, sizes=(8, 16, 24))
        mine = shard.frames_of_rank(cams, world, rank)
        # stand-in for each frame's rendered output: its index repeated per pixel
        per = {i: np.full(cams[i].x_pix * cams[i].y_pix, float(i), np.float32) for i in mine}
        got = shard.gather_frames(per, len(cams), world)
        # the weak-scaling timing rule of the bench: max over ranks
        import torch
        t = torch.tensor([float(rank + 1)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            result_q.put(([None if g is None else g.tolist() for g in got], float(t.item()),
                          [c.x_pix * c.y_pix for c in cams]))
    finally:
        dist.destroy_process_group()


def test_gather_frames_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, tmax, sizes = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert tmax == 2.0
    assert len(got) == 12
    for i, g in enumerate(got):
        assert len(g) == sizes[i] and all(v == i for v in g)
