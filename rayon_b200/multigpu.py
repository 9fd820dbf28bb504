"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host-side
exchange only (paths are independent, so no collective sits inside a render).

* Job sharding (serving across GPUs): jobs are dealt to ranks greedily by
  cost (pixels x samples), largest first, each to the least-loaded rank; every
  rank serves its shard with its own batched server; results are gathered on
  rank 0 only when asked.
* Sample split of one job: rank r renders samples [r*S/N, (r+1)*S/N) into its
  own accumulation (the counter-based streams make the union equal to a
  single-GPU render of all S samples); the per-pixel sums are then summed over
  ranks in FP64 (sum minus Kahan compensation, widened before the reduce).
"""
from __future__ import annotations

import numpy as np


def shard_jobs(costs, world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of job indices to `world` ranks."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    for o in out:
        o.sort()
    return out


def sample_range(spp: int, rank: int, world: int) -> tuple[int, int]:
    """[first, count) of the samples rank `rank` renders in a sample-split job."""
    base, extra = divmod(spp, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def reduce_accumulation(sum_comp, group=None):
    """Sum a Kahan (sum, compensation) accumulation over ranks in FP64.

    sum_comp: torch tensor (2, n, 4) float32 [sums; compensations] on this
    rank's device. Returns the (n, 3) float64 total on every rank."""
    import torch
    import torch.distributed as dist
    total = (sum_comp[0, :, :3].double() - sum_comp[1, :, :3].double()).contiguous()
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(total, op=dist.ReduceOp.SUM, group=group)
    return total


def gather_results(local: dict, group=None) -> dict:
    """All-gather {job index: array} dicts from every rank (host objects)."""
    import torch.distributed as dist
    if not (dist.is_initialized() and dist.get_world_size(group) > 1):
        return dict(local)
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, {k: np.asarray(v) for k, v in local.items()}, group=group)
    out: dict = {}
    for p in parts:
        out.update(p)
    return out
