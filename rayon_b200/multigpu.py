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


def _rank_world(group=None) -> tuple[int, int]:
    import torch.distributed as dist
    if dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def render_sample_split(render_range, spp: int, group=None):
    """One job split by samples over the ranks of `group`.

    render_range(first, count) renders samples [first, first + count) of the
    job on this rank's GPU and returns its accumulation as a (2, n, 4) float32
    tensor [sums; Kahan compensations] (gpu_range_renderer makes one over the
    per-frame kernel). Rank r takes sample_range(spp, r, world); the FP64 sums
    are all-reduced, so every rank returns the (n, 3) float64 sums of all spp
    samples: the same samples, and so the same image up to FP32 summation
    order, as one GPU rendering them all."""
    rank, world = _rank_world(group)
    first, count = sample_range(spp, rank, world)
    acc = render_range(first, count)
    return reduce_accumulation(acc, group)


def gpu_range_renderer(ds, frame, width: int, height: int, depth: int, background: float = 1.0, dof=None,
                       nee: bool = False, seed: int | None = None):
    """render_range for render_sample_split: rb_render_accumulate of the
    scene `ds` (uploaded on this rank's device) into a fresh (2, n, 4) buffer,
    on the sample streams of `seed` (render.DEFAULT_SEED when None, the
    streams of render.render_accumulate)."""
    import ctypes as C

    import torch

    from . import render
    from ._native import check, lib

    fr = np.ascontiguousarray(frame, np.float64)

    def run(first: int, count: int):
        acc = torch.zeros((2, width * height, 4), dtype=torch.float32, device="cuda")
        if count > 0:
            render.set_globals(background=background, dof=dof)
            with render.options(nee=nee, seed=render.DEFAULT_SEED if seed is None else seed):
                check(lib.rb_render_accumulate(ds.handle, width, height, fr.ctypes.data_as(C.POINTER(C.c_double)),
                                               count, first, depth, C.c_void_p(acc[0].data_ptr()),
                                               C.c_void_p(acc[1].data_ptr()), None,
                                               C.c_void_p(torch.cuda.current_stream().cuda_stream)),
                      "rb_render_accumulate")
            render.set_globals()
        return acc

    return run


def serve_sharded(costs, run_shard, group=None) -> dict:
    """A request stream served across the ranks of `group`, one server per
    rank. Jobs are dealt by shard_jobs(costs) (largest first, least-loaded
    rank); run_shard(indices) serves this rank's jobs on its GPU and returns
    {"latencies": {job index: seconds}, "paths": int, "seconds": float}
    (gpu_shard_runner makes one over rb_server). The per-rank results are
    all-gathered: every rank returns the latencies of all jobs, each rank's
    paths and seconds, and the aggregate Mpaths/s = all paths / the slowest
    rank's seconds."""
    import torch.distributed as dist
    rank, world = _rank_world(group)
    mine = shard_jobs(costs, world)[rank]
    res = run_shard(mine)
    out = {"latencies": dict(res["latencies"]), "paths": [int(res["paths"])], "seconds": [float(res["seconds"])],
           "shards": [list(mine)]}
    if world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, {"latencies": dict(res["latencies"]), "paths": int(res["paths"]),
                                       "seconds": float(res["seconds"]), "shard": list(mine)}, group=group)
        out = {"latencies": {}, "paths": [], "seconds": [], "shards": []}
        for p in parts:
            out["latencies"].update(p["latencies"])
            out["paths"].append(p["paths"])
            out["seconds"].append(p["seconds"])
            out["shards"].append(p["shard"])
    slowest = max(out["seconds"]) if out["seconds"] else 0.0
    out["mpaths_s"] = sum(out["paths"]) / slowest / 1e6 if slowest > 0 else None
    lat = np.array([out["latencies"][k] for k in sorted(out["latencies"])]) if out["latencies"] else np.zeros(0)
    out["p50_latency_s"] = float(np.percentile(lat, 50)) if lat.size else None
    out["p99_latency_s"] = float(np.percentile(lat, 99)) if lat.size else None
    return out


def gpu_shard_runner(device_scenes, requests, server_kwargs=None):
    """run_shard for serve_sharded: a serving.Server on this rank's GPU with the
    rank's own uploads of the scenes (device_scenes, in request scene order);
    requests[i] is job i's rb_job_request (its scene field indexes
    device_scenes). Runs the shard's jobs with their arrival times and
    reports latencies, paths and wall seconds."""
    import time

    from . import serving

    def run(indices):
        srv = serving.Server(**(server_kwargs or {}))
        ids = [srv.add_scene(ds) for ds in device_scenes]
        reqs = []
        for i in indices:
            r = type(requests[i]).from_buffer_copy(requests[i])   # the caller's request stays as it was
            r.scene = ids[r.scene]
            reqs.append(r)
        paths = sum(r.width * r.height * r.spp for r in reqs)
        t0 = time.time()
        lat = srv.run_trace(reqs, realtime=True) if reqs else np.zeros(0)
        secs = time.time() - t0
        srv.close()
        return {"latencies": {i: float(v) for i, v in zip(indices, lat)}, "paths": paths, "seconds": secs}

    return run
