"""Walker shards across ranks (one process per GPU).

Walkers are independent and a walker's random stream depends only on its
global id, so a job of world * n walkers splits into contiguous shards; the
only exchange is the final sum of the FP64 accumulators (sig0, dx2, dx4,
counts, signals), done here as an all-gather summed in rank order so the
result does not depend on message timing.
"""
from __future__ import annotations

import numpy as np


def walker_shard(per_rank: int, rank: int) -> tuple[int, int]:
    """[begin, end) walker ids of `rank` when every rank walks `per_rank`."""
    return rank * per_rank, (rank + 1) * per_rank


def split_range(npar: int, rank: int, world: int) -> tuple[int, int]:
    """[begin, end) of an npar-walker job split as evenly as possible."""
    return npar * rank // world, npar * (rank + 1) // world


def gather_sum(fields: dict, group=None, device=None) -> dict:
    """Sum per-rank result fields (numpy arrays) over all ranks, in rank order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    keys = sorted(fields)
    flat = np.concatenate([np.asarray(fields[k], dtype=np.float64).ravel() for k in keys])
    t = torch.from_numpy(flat)
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    total = parts[0].clone()
    for p in parts[1:]:
        total += p
    total = total.cpu().numpy()
    out, off = {}, 0
    for k in keys:
        a = np.asarray(fields[k])
        out[k] = total[off:off + a.size].reshape(a.shape)
        off += a.size
    return out
