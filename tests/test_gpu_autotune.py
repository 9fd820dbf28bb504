"""The autotuner (RB_LAYOUT_AUTOTUNE): layout and leaf size, the per-frame
kernel's register budget and block shape, the traversal stack's shared-memory
depth and, for smooth-SDF scenes, the wavefront engine's path slots; decisions
cached per (GPU, scene fingerprint), reused without probing by a second
upload, and the reused decision renders the same image bit for bit."""
import numpy as np
import pytest

from rayon_b200 import render, scenes

pytestmark = pytest.mark.gpu


def test_decision_is_cached_and_renders_the_same(cuda):
    spec = scenes.one_weekend(seed=777, width=160, height=90, spp=16)   # a scene no other test tunes
    sc = spec.to_scene()
    sc.build_bvh()
    fr = spec.camera.frame(160, 90)
    a = sc.upload(layout="autotune", tune_depth=spec.depth, probe=(fr, 160, 90))
    ta = a.tuning
    assert ta["from_cache"] == 0 and ta["probe_ms"] > 0
    assert ta["blocks_per_sm"] in (2, 3, 4)
    assert (ta["block_x"], ta["block_y"]) in ((8, 8), (16, 8), (16, 16), (32, 8))
    assert ta["short_stack"] in (4, 8, 16)
    assert ta["wavefront_queue"] == 0            # no smooth SDF field
    b = sc.upload(layout="autotune", tune_depth=spec.depth, probe=(fr, 160, 90))
    tb = b.tuning
    assert tb["from_cache"] == 1
    assert {k: v for k, v in ta.items() if k != "from_cache"} == {k: v for k, v in tb.items() if k != "from_cache"}
    ia = render.render_accumulate(a, fr, 160, 90, 16, spec.depth, background=1.0, dof=spec.dof)
    ib = render.render_accumulate(b, fr, 160, 90, 16, spec.depth, background=1.0, dof=spec.dof)
    np.testing.assert_array_equal(ia, ib)
    # and the tuned configuration renders what the class defaults render (same samples)
    d = sc.upload()
    idf = render.render_accumulate(d, fr, 160, 90, 16, spec.depth, background=1.0, dof=spec.dof)
    bad = (np.abs(ia - idf) > 1e-3 * (1 + np.abs(idf)) * 16).any(axis=2)
    assert bad.mean() < 0.01
    for ds in (a, b, d):
        ds.free()


def test_smooth_sdf_scene_gets_a_wavefront_queue_depth(cuda):
    spec = scenes.sdf_field(seed=99, count=32, width=96, height=54, spp=4, depth=4)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload(layout="autotune", tune_depth=spec.depth)
    t = ds.tuning
    assert t["wavefront_queue"] in (1 << 21, 1 << 22, 1 << 23, 1 << 24)
    fr = spec.camera.frame(96, 54)
    a = render.render_wavefront(ds, fr, 96, 54, 4, spec.depth)                  # the tuned capacity
    b = render.render_wavefront(ds, fr, 96, 54, 4, spec.depth, queue_capacity=1 << 20)
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9)
    ds.free()
