"""Multi-GPU sharding: one process per GPU. Batched renders shard by frame;
one frame shards by interleaved tile x tile pixel tiles (tile t -> rank t mod
world, which spreads the expensive photon-ring pixels over the ranks), each
tile a windowed camera, a rank's tiles rendered in one batched launch. Rays are
independent; the only exchange is the gather of each rank's finished frames or
tiles to rank 0. torch.distributed carries the gather (NCCL on GPUs, gloo on
CPU).
"""
from __future__ import annotations

import math

import numpy as np


def frame_cost(x_pix: int, y_pix: int, tol: float) -> float:
    """Relative cost estimate of a frame: rays x (1/tol)^(1/5), the growth of a
    5th-order method's step count with the tolerance."""
    return float(x_pix) * float(y_pix) * (1.0 / tol) ** 0.2


def assign_frames(costs, world: int) -> list:
    """Greedy longest-processing-time assignment of frames to ranks; returns,
    per rank, the ascending list of frame indices it renders."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(v) for v in out]


def frames_of_rank(cams, world: int, rank: int) -> list:
    costs = [frame_cost(c.x_pix, c.y_pix if c.y_pix else c.x_pix, c.tolerance) for c in cams]
    return assign_frames(costs, world)[rank]


def gather_frames(per_frame: dict, n_frames: int, world: int, group=None) -> list | None:
    """All ranks pass {frame index: 1-D float32 array}; rank 0 receives the list
    of every frame's array in frame order (other ranks get None). One
    all-reduce (max) of the per-rank sizes, gather_object of the (small)
    index/size metadata to rank 0, and one gather of a padded float32 tensor
    to rank 0: the data crosses the links once, to the rank that assembles it."""
    import torch
    import torch.distributed as dist

    if world == 1:
        return [per_frame[i] for i in range(n_frames)]
    rank = dist.get_rank(group)
    meta = [(i, int(a.size)) for i, a in sorted(per_frame.items())]
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    size = torch.tensor([sum(s for _, s in meta)], dtype=torch.int64, device=dev)
    dist.all_reduce(size, op=dist.ReduceOp.MAX, group=group)
    cap = max(int(size.item()), 1)
    metas = [None] * world if rank == 0 else None
    dist.gather_object(meta, metas, dst=0, group=group)
    buf = torch.zeros(cap, dtype=torch.float32, device=dev)
    flat = np.concatenate([per_frame[i] for i, _ in meta]).astype(np.float32) if meta else np.zeros(0, np.float32)
    buf[: flat.size] = torch.from_numpy(flat).to(dev)
    bufs = [torch.empty(cap, dtype=torch.float32, device=dev) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, bufs, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * n_frames
    for r, m in enumerate(metas):
        data = bufs[r].cpu().numpy()
        off = 0
        for i, s in m:
            out[i] = data[off:off + s].copy()
            off += s
    return out


def balance(costs, assignment) -> float:
    """max rank load / mean rank load (1.0 is perfect)."""
    loads = [sum(costs[i] for i in a) for a in assignment]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def tile_windows(x_pix: int, y_pix: int, tile: int = 16) -> list:
    """(x0, y0, w, h) of the image's tile x tile tiles, row-major (edge tiles
    are cut to the image)."""
    return [(x0, y0, min(tile, x_pix - x0), min(tile, y_pix - y0))
            for y0 in range(0, y_pix, tile) for x0 in range(0, x_pix, tile)]


def tiles_of_rank(n_tiles: int, world: int, rank: int) -> list:
    """Interleaved tiles: tile t goes to rank t mod world."""
    return list(range(rank, n_tiles, world))


# per-pixel width of each gathered field
_WIDTH = {"xyz": 3, "class": 1, "steps": 1}


def assemble_tiles(wins, tiles: dict, x_pix: int, y_pix: int, want=("xyz", "class", "steps")) -> dict:
    """{tile index: {field: array of the tile's pixels, row-major}} -> whole-
    image arrays indexed by pixel i + x_pix * j (every tile of wins present)."""
    out = {}
    for k in want:
        wdt = _WIDTH[k]
        img = None
        for t, (x0, y0, w, h) in enumerate(wins):
            a = np.asarray(tiles[t][k])
            if img is None:
                img = np.zeros((y_pix, x_pix, wdt), dtype=a.dtype)
            img[y0:y0 + h, x0:x0 + w, :] = a.reshape(h, w, wdt)
        out[k] = img.reshape(y_pix * x_pix, wdt) if wdt > 1 else img.reshape(y_pix * x_pix)
    return out


def render_frame_tiles(renderer, scene, cam, colors, world: int = 1, rank: int = 0, tile: int = 16,
                       want=("xyz", "class", "steps"), group=None, **kw):
    """One frame split over `world` ranks in interleaved tile x tile tiles: this
    rank renders its tiles as windowed cameras in batched launches (at most
    RTW_MAX_FRAMES windows each); rank 0 returns the whole frame's arrays
    (pixel i + x_pix * j), the other ranks None. The arrays equal those of a
    render of the whole frame (each ray's arithmetic does not depend on its
    batch)."""
    from . import abi

    abi.camera_pixels(cam)
    wins = tile_windows(cam.x_pix, cam.y_pix, tile)
    mine = tiles_of_rank(len(wins), world, rank)
    tiles = {}
    for b in range(0, len(mine), abi.MAX_FRAMES):
        chunk = mine[b:b + abi.MAX_FRAMES]
        res = renderer.render(scene, [abi.window(cam, *wins[t]) for t in chunk], colors, want=want, **kw)
        off = 0
        for t in chunk:
            n = wins[t][2] * wins[t][3]
            tiles[t] = {k: res[k][off:off + n] for k in want}
            off += n
    if world == 1:
        return assemble_tiles(wins, tiles, cam.x_pix, cam.y_pix, want)
    # one float32 array per tile: the fields one after another (classes and
    # step counts below 2^24 are exact in float32)
    flat = {t: np.concatenate([np.asarray(v[k], np.float64).ravel() for k in want]).astype(np.float32)
            for t, v in tiles.items()}
    got = gather_frames(flat, len(wins), world, group=group)
    if got is None:
        return None
    dtypes = {"xyz": np.float32, "class": np.uint8, "steps": np.uint32}
    back = {}
    for t, (x0, y0, w, h) in enumerate(wins):
        n, off, d = w * h, 0, {}
        for k in want:
            m = n * _WIDTH[k]
            d[k] = got[t][off:off + m].astype(dtypes[k])
            off += m
        back[t] = d
    return assemble_tiles(wins, back, cam.x_pix, cam.y_pix, want)


__all__ = ["frame_cost", "assign_frames", "frames_of_rank", "gather_frames", "balance", "tile_windows",
           "tiles_of_rank", "assemble_tiles", "render_frame_tiles", "math"]
