"""Multi-GPU sharding of batched renders: one process per GPU, frames as the
shard unit (rays are independent; the only exchange is the gather of each
rank's finished frames). torch.distributed carries the gather (NCCL on GPUs,
gloo on CPU).
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
    of every frame's array in frame order (other ranks get None). Uses
    all_gather_object for the (small) index/size metadata and one
    all_gather of a padded float32 tensor for the data."""
    import torch
    import torch.distributed as dist

    if world == 1:
        return [per_frame[i] for i in range(n_frames)]
    rank = dist.get_rank(group)
    meta = [(i, int(a.size)) for i, a in sorted(per_frame.items())]
    metas = [None] * world
    dist.all_gather_object(metas, meta, group=group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    sizes = [sum(s for _, s in m) for m in metas]
    cap = max(max(sizes), 1)
    buf = torch.zeros(cap, dtype=torch.float32, device=dev)
    flat = np.concatenate([per_frame[i] for i, _ in meta]).astype(np.float32) if meta else np.zeros(0, np.float32)
    buf[: flat.size] = torch.from_numpy(flat).to(dev)
    bufs = [torch.empty(cap, dtype=torch.float32, device=dev) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
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


__all__ = ["frame_cost", "assign_frames", "frames_of_rank", "gather_frames", "balance", "math"]
