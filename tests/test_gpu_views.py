"""Several views in one persistent launch (rb_render_views): view 0 repeats
the per-frame kernel's sample streams, every view agrees with the per-frame
kernel on its own salt's streams through the server, and the counters add up."""
import numpy as np
import pytest

from rayon_b200 import render, scenes, serving

pytestmark = pytest.mark.gpu


def _orbit_frames(spec, n, w, h):
    return [scenes.orbit(spec.camera, 2 * np.pi * v / n).frame(w, h) for v in range(n)]


def _paired(a, b, spp, name):
    """Same sample streams. Triangle scenes agree pixel for pixel; on the
    smooth SDF field the two kernels (compiled separately) may round a march
    step differently in the last bit, and a path that then branches
    differently changes its pixel, so a few pixels may differ (the paired
    tolerance of the other SDF engine comparisons) while the images agree."""
    if name != "sdf_field":
        np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-4 * spp)
        return
    bad = (np.abs(a - b) > 1e-4 * (1 + np.abs(b)) * spp).any(axis=-1)
    assert bad.mean() < 0.01, bad.mean()
    np.testing.assert_allclose(a.mean((0, 1)), b.mean((0, 1)), rtol=1e-2)


@pytest.mark.parametrize("name", ["cornell", "sdf_field"])
def test_views_match_single_frames(cuda, name):
    spec = scenes.sdf_field(count=48) if name == "sdf_field" else scenes.cornell()
    w, h, spp, n = 48, 32, 16, 5
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    frames = _orbit_frames(spec, n, w, h)
    imgs, cnt = render.render_views(ds, frames, w, h, spp, spec.depth, background=spec.background, counters=True)
    assert imgs.shape == (n, h, w, 3) and np.isfinite(imgs).all()
    assert cnt[1] == n * w * h * spp and cnt[0] >= cnt[1]
    # view 0 draws salt 0, the streams of rb_render_accumulate
    ref0 = render.render_accumulate(ds, frames[0], w, h, spp, spec.depth, background=spec.background)
    _paired(imgs[0], ref0, spp, name)
    # view v draws salt v: the server's job with seed (salt) v
    srv = serving.Server(paths_per_iteration=1 << 24, max_spp_per_iteration=spp)
    sid = srv.add_scene(ds)
    for v in range(1, n):
        j = srv.submit(serving.job(sid, frames[v], w, h, spp, spec.depth, background=spec.background, seed=v))
        srv.drain()
        _paired(imgs[v], srv.fetch(j, w, h), spp, name)
    srv.close()
    ds.free()


def test_views_accumulate_and_reject_bad_arguments(cuda):
    import ctypes as C
    import torch
    from rayon_b200 import lib
    spec = scenes.cornell()
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    w, h = 32, 32
    frames = _orbit_frames(spec, 3, w, h)
    a = render.render_views(ds, frames, w, h, 8, spec.depth, background=0.0)
    b = render.render_views(ds, frames, w, h, 8, spec.depth, background=0.0, sample_base=8)
    both = render.render_views(ds, frames, w, h, 16, spec.depth, background=0.0)
    np.testing.assert_allclose(a + b, both, rtol=1e-4, atol=2e-3)
    fr = np.ascontiguousarray(np.stack(frames))
    acc = torch.zeros((3, 2, w * h, 4), device="cuda")
    for bad in ((0, w, h), (3, 0, h), (3, w, -1)):
        st = lib.rb_render_views(ds.handle, bad[0], bad[1], bad[2], fr.ctypes.data_as(C.POINTER(C.c_double)), 4, 0,
                                 4, C.c_void_p(acc.data_ptr()), None, None)
        assert st < 0
    ds.free()


@pytest.mark.parametrize("name", ["cornell", "sdf_field"])
def test_views_wavefront_paired_with_views_kernel(cuda, name):
    # one wavefront run over all views draws the same streams (view v on salt
    # v) as the batched kernel; the paths agree except where FP32 marching or
    # accumulation order branches a path differently
    spec = scenes.sdf_field(count=48) if name == "sdf_field" else scenes.cornell()
    w, h, spp, n = 48, 32, 8, 4
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    frames = _orbit_frames(spec, n, w, h)
    a = render.render_views(ds, frames, w, h, spp, spec.depth, background=spec.background)
    b, cnt = render.render_views_wavefront(ds, frames, w, h, spp, spec.depth, background=spec.background,
                                           queue_capacity=2048, counters=True)
    assert int(cnt[1]) == n * w * h * spp
    bad = (np.abs(a - b) > 2e-3 * (1 + np.abs(a)) * spp).any(axis=3)
    assert bad.mean() < 0.04, bad.mean()
    np.testing.assert_allclose(a.mean((1, 2)), b.mean((1, 2)), rtol=2e-2, atol=1e-3)
    ds.free()
