"""Failure paths, made on the host or by a bounded loop, never by faulting the
GPU: the BVH traversal's step budget (which no well-formed tree reaches) is
counted per scene when it runs out, and device-allocation failures injected on
the host (rb_inject_alloc_failures) reject one served job with
RB_ERR_OUT_OF_MEMORY while the server keeps serving, and make one wavefront
run fail cleanly after which the engine allocates afresh."""
import numpy as np
import pytest

from rayon_b200 import lib, render, scenes, serving

pytestmark = pytest.mark.gpu
RB_ERR_OUT_OF_MEMORY, RB_ERR_CAPACITY = -3, -5


@pytest.mark.parametrize("name", ["cornell", "one_weekend"])
def test_well_formed_tree_has_no_traversal_faults(cuda, name):
    spec = getattr(scenes, name)(width=96, height=64, spp=8)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    render.render_accumulate(ds, spec.camera.frame(96, 64), 96, 64, 8, spec.depth, background=spec.background,
                             dof=spec.dof)
    assert ds.traversal_faults() == 0
    ds.free()


def test_budget_exhaustion_is_counted_and_reset(cuda):
    spec = scenes.one_weekend(width=64, height=36, spp=2)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload(traversal_budget=3)      # a budget far below the tree's depth
    img = render.render_accumulate(ds, spec.camera.frame(64, 36), 64, 36, 2, spec.depth, background=1.0)
    assert np.isfinite(img).all()          # the loop stops, the ray keeps what it found
    n = ds.traversal_faults(reset=True)
    assert n > 64 * 36 // 2
    assert ds.traversal_faults() == 0
    ds.free()


def test_server_rejects_job_on_allocation_failure_and_keeps_serving(cuda):
    spec = scenes.cornell()
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    srv = serving.Server()
    sid = srv.add_scene(ds)
    reqs = [serving.job(sid, spec.camera.frame(w, w), w, w, 16, spec.depth, background=0.0, seed=k)
            for k, w in enumerate((64, 48, 80))]
    try:
        assert lib.rb_inject_alloc_failures(b"server_job", 1) == 0
        ids = [srv.submit(r) for r in reqs]
        srv.drain()
        st = [srv.status(i) for i in ids]
        assert st[0].state == -1 and st[0].error == RB_ERR_OUT_OF_MEMORY
        assert [s.state for s in st[1:]] == [2, 2] and [s.error for s in st[1:]] == [0, 0]
        assert srv.stats().jobs_rejected == 1
        # the served results are the jobs' own: same as the job alone on a fresh server
        alone = serving.Server()
        a_sid = alone.add_scene(ds)
        j = alone.submit(serving.job(a_sid, spec.camera.frame(48, 48), 48, 48, 16, spec.depth, background=0.0,
                                     seed=1))
        alone.drain()
        np.testing.assert_allclose(srv.fetch(ids[1], 48, 48), alone.fetch(j, 48, 48), rtol=2e-5, atol=4e-4)
        alone.close()
        # and it keeps admitting
        k = srv.submit(reqs[0])
        srv.drain()
        assert srv.status(k).state == 2
    finally:
        lib.rb_inject_alloc_failures(b"server_job", 0)
        srv.close()
        ds.free()


def test_wavefront_queue_allocation_failure_then_recovery(cuda):
    spec = scenes.cornell(width=48, height=48, spp=4)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(48, 48)
    cap = (1 << 18) + 4096                 # a capacity no other test uses: the engine must allocate
    try:
        assert lib.rb_inject_alloc_failures(b"wavefront_queue", 1) == 0
        with pytest.raises(RuntimeError, match="out of memory|rb_render_wavefront"):
            render.render_wavefront(ds, fr, 48, 48, 4, spec.depth, background=0.0, queue_capacity=cap)
        a = render.render_wavefront(ds, fr, 48, 48, 4, spec.depth, background=0.0, queue_capacity=cap)
        b = render.render_wavefront(ds, fr, 48, 48, 4, spec.depth, background=0.0, queue_capacity=1 << 20)
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9)   # same samples, FP64 sums
        assert a.mean() > 0
    finally:
        lib.rb_inject_alloc_failures(b"wavefront_queue", 0)
        ds.free()
