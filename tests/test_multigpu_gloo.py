"""Host-side multi-GPU logic on CPU with two gloo ranks (no GPU): job sharding
covers every job once and balances cost, sample ranges tile [0, spp), and the
FP64 reduction of Kahan accumulations equals the single-process sum."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from rayon_b200 import multigpu


def test_shard_jobs_balanced_and_complete():
    rng = np.random.default_rng(0)
    costs = list(rng.integers(1, 1000, 37).astype(float))
    for world in (1, 2, 3, 8):
        sh = multigpu.shard_jobs(costs, world)
        allj = sorted(i for s in sh for i in s)
        assert allj == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in sh]
        assert max(loads) - min(loads) <= max(costs)


def test_sample_ranges_tile():
    for spp in (1, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                f, n = multigpu.sample_range(spp, r, world)
                got += list(range(f, f + n))
            assert got == list(range(spp))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _fake_range(first, count, npx):
    """A stand-in for one rank's render of samples [first, first + count):
    sample s adds pixel % 7 + 0.5 s to every channel (exact in FP32)."""
    pix = torch.arange(npx, dtype=torch.float32)
    acc = torch.zeros((2, npx, 4), dtype=torch.float32)
    for s in range(first, first + count):
        acc[0, :, :3] += (pix % 7 + 0.5 * s)[:, None]
    return acc


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 100
        g = torch.Generator().manual_seed(1234)
        full = torch.rand((world, 2, n, 4), generator=g, dtype=torch.float32)
        full[:, 1] *= 1e-6  # small compensation terms
        mine = full[rank].clone()
        tot = multigpu.reduce_accumulation(mine)
        expect = (full[:, 0, :, :3].double() - full[:, 1, :, :3].double()).sum(0)
        ok_reduce = torch.allclose(tot, expect, rtol=0, atol=1e-12)
        costs = [float(c) for c in range(1, 11)]
        shard = multigpu.shard_jobs(costs, world)[rank]
        res = multigpu.gather_results({i: np.full(3, i, np.float32) for i in shard})
        ok_gather = sorted(res) == list(range(10)) and all(float(res[i][0]) == i for i in res)
        # sample split: each rank renders only its range; the reduce gives the
        # single-process sums of all samples (values exact in FP32)
        spp, npx = 37, 50
        total = multigpu.render_sample_split(lambda f, c: _fake_range(f, c, npx), spp)
        ok_split = torch.equal(total, _fake_range(0, spp, npx)[0, :, :3].double())
        # sharded serving: every job served once, stats gathered on every rank
        jc = [float(c) for c in (5, 1, 9, 3, 7, 2, 8)]
        out = multigpu.serve_sharded(jc, lambda idx: {"latencies": {i: 0.5 * i for i in idx},
                                                      "paths": int(sum(jc[i] for i in idx)),
                                                      "seconds": 1.0 + rank})
        ok_serve = (sorted(out["latencies"]) == list(range(len(jc))) and
                    sorted(i for sh in out["shards"] for i in sh) == list(range(len(jc))) and
                    sum(out["paths"]) == int(sum(jc)) and abs(out["mpaths_s"] - sum(jc) / world / 1e6) < 1e-12)
        q.put((rank, ok_reduce, ok_gather and ok_split and ok_serve))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(r[1] and r[2] for r in out), out
