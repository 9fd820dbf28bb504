"""The multi-GPU drivers with the real kernels on one GPU: a sample-split
render (rank ranges rendered one after another here, then summed in FP64)
gives the single-launch image, and the sharded-serving runner serves every job
of its shard. Ranks that wait on one another are not emulated: the ranges are
independent renders. The collectives themselves are covered by the
world-size-2 gloo tests."""
import numpy as np
import pytest

from rayon_b200 import multigpu, render, scenes, serving

pytestmark = pytest.mark.gpu


def _cornell(w=64, h=64):
    spec = scenes.cornell(width=w, height=h, spp=24)
    sc = spec.to_scene()
    sc.build_bvh()
    return spec, sc.upload()


def test_sample_split_equals_single_render(cuda):
    spec, ds = _cornell()
    fr = spec.camera.frame(64, 64)
    run = multigpu.gpu_range_renderer(ds, fr, 64, 64, spec.depth, background=0.0)
    one = multigpu.render_sample_split(run, 24).cpu().numpy()        # no process group: one rank
    ref = render.render_accumulate(ds, fr, 64, 64, 24, spec.depth, background=0.0).reshape(-1, 3)
    np.testing.assert_allclose(one, ref, rtol=1e-6, atol=1e-6)
    # three ranks' ranges, rendered independently and summed in FP64
    parts = []
    for r in range(3):
        f, c = multigpu.sample_range(24, r, 3)
        a = run(f, c)
        parts.append((a[0, :, :3].double() - a[1, :, :3].double()).cpu().numpy())
    np.testing.assert_allclose(sum(parts), ref, rtol=2e-5, atol=2e-5 * 24)
    ds.free()


def test_sharded_serving_runner_serves_its_shard(cuda):
    spec, ds = _cornell()
    reqs = [serving.job(0, spec.camera.frame(w, w), w, w, s, spec.depth, background=0.0, seed=k, arrival=0.01 * k)
            for k, (w, s) in enumerate([(64, 16), (32, 64), (48, 8), (80, 4), (40, 32)])]
    costs = [r.width * r.height * r.spp for r in reqs]
    out = multigpu.serve_sharded(costs, multigpu.gpu_shard_runner([ds], reqs))
    assert sorted(out["latencies"]) == list(range(5))
    assert all(v > 0 for v in out["latencies"].values())
    assert out["paths"] == [sum(costs)] and out["mpaths_s"] > 0
    assert [r.scene for r in reqs] == [0] * 5          # the caller's requests are untouched
    ds.free()
