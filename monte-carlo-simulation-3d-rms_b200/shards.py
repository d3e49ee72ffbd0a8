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


# rms_adjoint_run's outputs that are sums over walkers: a shard's values add up
# to the whole job's (dL/dwave, D by time rescaling and pathwise, kappa by
# forced draws, T2, the loss and the signal sums)
ADJOINT_SUMS = ("d_wave", "d_diffusivity", "d_diffusivity_pathwise", "d_kappa", "d_t2", "loss", "sigw")


def adjoint_sum(grads: dict, group=None, device=None) -> dict:
    """The whole job's adjoint from one rank's walker shard (Sim.adjoint with
    walker_range = that shard): every walker sum added over ranks in rank
    order.  d_kappa_score, whose baseline is the shard's own mean loss, is
    summed too: the sum of the shards' score estimates, unbiased like each of
    them, though not the single run's value.  Every rank passes the same
    keys (the fields present in grads are summed)."""
    fields = {k: np.asarray(grads[k], dtype=np.float64) for k in ADJOINT_SUMS + ("d_kappa_score",) if k in grads}
    tot = gather_sum(fields, group=group, device=device)
    out = dict(grads)
    for k, v in tot.items():
        out[k] = float(v) if np.ndim(grads[k]) == 0 else v
    return out

