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


# ---- one frame over ranks in interleaved tiles ---------------------------

@pytest.mark.parametrize("x_pix,y_pix,tile", [(64, 45, 16), (17, 3, 16), (100, 71, 8), (1, 1, 16)])
def test_tiles_cover_the_image_once(x_pix, y_pix, tile):
    wins = shard.tile_windows(x_pix, y_pix, tile)
    hit = np.zeros((y_pix, x_pix), int)
    for x0, y0, w, h in wins:
        assert 1 <= w <= tile and 1 <= h <= tile
        hit[y0:y0 + h, x0:x0 + w] += 1
    assert np.all(hit == 1)
    for world in (1, 2, 3, 8):
        parts = [shard.tiles_of_rank(len(wins), world, r) for r in range(world)]
        assert sorted(t for p in parts for t in p) == list(range(len(wins)))


class _FakeRenderer:
    """Stands in for Renderer.render on the CPU: each windowed camera's pixels
    get values made from their whole-image coordinates (i, j)."""

    def render(self, scene, cams, colors, want=("xyz", "class", "steps"), **kw):
        out = {k: [] for k in want}
        for c in cams:
            j, i = np.mgrid[c.win_y0:c.win_y0 + c.win_h, c.win_x0:c.win_x0 + c.win_w]
            i, j = i.ravel(), j.ravel()
            out["xyz"].append(np.stack([i, j, i + 2 * j], 1).astype(np.float32))
            out["class"].append(((i + j) % 7).astype(np.uint8))
            out["steps"].append((1000 * i + j).astype(np.uint32))
        return {k: np.concatenate(v) for k, v in out.items()}


def _expected(x_pix, y_pix):
    j, i = np.mgrid[0:y_pix, 0:x_pix]
    i, j = i.ravel(), j.ravel()
    return {"xyz": np.stack([i, j, i + 2 * j], 1).astype(np.float32), "class": ((i + j) % 7).astype(np.uint8),
            "steps": (1000 * i + j).astype(np.uint32)}


def test_render_frame_tiles_one_rank():
    from rtwca_b200 import abi
    cam = abi.make_camera([0, 25, 1.0, 0], x_pix=37)
    got = shard.render_frame_tiles(_FakeRenderer(), None, cam, [500.0], world=1, rank=0, tile=8)
    exp = _expected(cam.x_pix, cam.y_pix)
    for k in exp:
        assert np.array_equal(got[k], exp[k]), k


def _tile_worker(rank, world, port, result_q):
    import torch.distributed as dist
    from rtwca_b200 import abi
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cam = abi.make_camera([0, 25, 1.0, 0], x_pix=45)
        got = shard.render_frame_tiles(_FakeRenderer(), None, cam, [500.0], world=world, rank=rank, tile=16)
        if rank == 0:
            exp = _expected(cam.x_pix, cam.y_pix)
            result_q.put(all(np.array_equal(got[k], exp[k]) for k in exp))
        else:
            result_q.put(got is None)
    finally:
        dist.destroy_process_group()


def test_render_frame_tiles_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_tile_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    oks = [q.get(timeout=120), q.get(timeout=120)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(oks)
