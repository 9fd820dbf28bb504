"""Radiance parity of the CUDA path tracer against the FP64 oracle on the same
counter-based sample streams (paired per path), estimator consistency (NEE vs
BSDF-only), Kahan accumulation, and the reference's own CUDA images (RMSE)."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from cases import HIT_CASES, REFIMG_CASES, mixed_materials  # noqa: E402

from oracle.oracle import Globals, OracleScene  # noqa: E402
from rayon_b200 import render, scenes  # noqa: E402

GOLDEN = Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu

# Paired tolerance: a pixel agrees when |gpu - oracle| <= 1e-3 * (1 + |oracle|) * spp.
# FP32 vs FP64 only breaks the pairing where a path takes a different branch
# (Russian roulette threshold, refract/reflect choice, grazing hit); at most
# this fraction of pixels may contain such a path.
MAX_DIVERGED = 0.03


def _cases():
    return {
        "cornell": (scenes.cornell(width=64, height=64), 16),
        "mixed_materials": (mixed_materials(), 16),
        "one_weekend": (scenes.one_weekend(width=120, height=68), 8),
        "small_icospheres": (HIT_CASES["small_icospheres"][0](), 4),
    }


def _render_pair(spec, spp, nee=False, width=None, height=None):
    w, h = width or spec.width, height or spec.height
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(w, h)
    img = render.render_accumulate(ds, fr, w, h, spp, spec.depth, background=spec.background, dof=spec.dof, nee=nee)
    g = Globals(background=spec.background, dof=spec.dof is not None,
                aperture=spec.dof[0] if spec.dof else 0.1, focus=spec.dof[1] if spec.dof else 10.0, nee=nee)
    ref, cnt = OracleScene(sc).render(fr, w, h, spp, spec.depth, g, seed=render.DEFAULT_SEED)
    ds.free()
    return img, ref.reshape(h, w, 3), cnt


@pytest.mark.parametrize("name", ["cornell", "mixed_materials", "one_weekend", "small_icospheres"])
@pytest.mark.parametrize("nee", [False, True])
def test_paired_radiance_vs_oracle(cuda, name, nee):
    spec, spp = _cases()[name]
    img, ref, _ = _render_pair(spec, spp, nee=nee)
    assert np.isfinite(img).all()
    bad = (np.abs(img - ref) > 1e-3 * (1 + np.abs(ref)) * spp).any(axis=2)
    assert bad.mean() < MAX_DIVERGED, f"{bad.mean():.4f} of pixels diverged"
    # image means agree tightly (divergent paths are rare and unbiased)
    np.testing.assert_allclose(img.mean((0, 1)), ref.mean((0, 1)), rtol=2e-2, atol=1e-3)


def test_nee_same_expectation(cuda):
    spec = scenes.cornell(width=32, height=32)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(32, 32)
    spp = 2048
    a = render.render_accumulate(ds, fr, 32, 32, spp, spec.depth, background=0.0, nee=False) / spp
    b = render.render_accumulate(ds, fr, 32, 32, spp, spec.depth, background=0.0, nee=True, sample_base=spp) / spp
    # whole-image mean radiance: same integral, two estimators
    ma, mb = a.mean(), b.mean()
    assert abs(ma - mb) / mb < 0.02, (ma, mb)
    # NEE lowers the variance: its per-pixel spread between two seeds is smaller
    b2 = render.render_accumulate(ds, fr, 32, 32, spp, spec.depth, background=0.0, nee=True, sample_base=3 * spp) / spp
    a2 = render.render_accumulate(ds, fr, 32, 32, spp, spec.depth, background=0.0, nee=False, sample_base=5 * spp) / spp
    assert np.sqrt(((b - b2) ** 2).mean()) < np.sqrt(((a - a2) ** 2).mean())
    ds.free()


def test_kahan_accumulation_beats_naive(cuda):
    spec = scenes.cornell(width=16, height=16)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(16, 16)
    spp = 8192
    k = render.render_accumulate(ds, fr, 16, 16, spp, 4, background=0.0, kahan=True)
    n = render.render_accumulate(ds, fr, 16, 16, spp, 4, background=0.0, kahan=False)
    ref, _ = OracleScene(sc).render(fr, 16, 16, spp, 4, Globals(background=0.0), seed=render.DEFAULT_SEED)
    ref = ref.reshape(16, 16, 3)
    ek = np.abs(k - ref).sum()
    en = np.abs(n - ref).sum()
    assert ek <= en
    ds.free()


def test_dropin_chunks_equal_single_launch(cuda):
    spec = scenes.cornell(width=40, height=40)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(40, 40)
    render.set_globals(background=0.0)
    a = render.render_dropin(ds, fr, 40, 40, 20, spec.depth, chunks=5)
    b = render.render_accumulate(ds, fr, 40, 40, 20, spec.depth, background=0.0)
    render.set_globals()
    # same sample indices, same Kahan state carried across calls
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6)
    ds.free()


def test_invisible_geometry_passes_camera_rays(cuda):
    # an invisible quad in front of a red sphere: camera rays pass through it at
    # bounce 0 (cuda_raytracer.cuh:879-883), so the centre pixel is red
    from rayon_b200 import scene as S
    sc = S.SceneDescription()
    red = sc.add_material(S.constant((1, 0, 0)))
    blue = sc.add_material(S.constant((0, 0, 1)))
    sc.add_sphere((0, 0, -5), 1.0, red)
    q = sc.add_rectangle((-1, -1, -2), (2, 0, 0), (0, 2, 0), blue)
    sc.set_visible(q, False)
    sc.build_bvh()
    ds = sc.upload()
    fr = S.camera_frame((0, 0, 0), (0, 0, -1), (0, 1, 0), 30.0, 9, 9)
    img = render.render_accumulate(ds, fr, 9, 9, 4, 4, background=0.0)
    np.testing.assert_allclose(img[4, 4] / 4, [1, 0, 0], atol=1e-6)
    # visible again: the quad is what the camera sees
    sc.set_visible(q, True)
    ds2 = sc.upload()
    img = render.render_accumulate(ds2, fr, 9, 9, 4, 4, background=0.0)
    np.testing.assert_allclose(img[4, 4] / 4, [0, 0, 1], atol=1e-6)
    ds.free()
    ds2.free()


@pytest.mark.parametrize("name", ["cornell", "mixed_materials", "one_weekend", "icospheres8"])
def test_converged_image_rmse_vs_reference_cuda(cuda, name):
    """Converged images against the reference's own CUDA renders
    (renderPixelsCUDAAccumulative at 2048-4096 spp, fixtures from
    make_golden.py --gpu): the One-Weekend configuration at full size with
    depth of field, a reduced icosphere set (8 level-5 GGX icospheres), the
    Cornell box and a scene with every material kind."""
    f = GOLDEN / f"refimg_{name}.npz"
    if not f.exists():
        pytest.skip("reference image fixture not generated")
    g = np.load(f)
    w, h, spp, depth = int(g["width"]), int(g["height"]), int(g["spp"]), int(g["depth"])
    spec = REFIMG_CASES[name][0]()
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(w, h)
    a = render.render_accumulate(ds, fr, w, h, spp, depth, background=spec.background, dof=spec.dof) / spp
    b = render.render_accumulate(ds, fr, w, h, spp, depth, background=spec.background, dof=spec.dof,
                                 sample_base=spp) / spp
    ref = g["sum"].astype(np.float64) / spp if "sum" in g else g["mean"].astype(np.float64)
    noise = np.sqrt(((a - b) ** 2).mean())          # two independent renders of ours
    err = np.sqrt(((a - ref) ** 2).mean())           # ours vs the reference renderer
    # same expectation => the cross RMSE is the noise RMSE, up to sampling scatter
    assert err < 1.35 * noise + 1e-4, (err, noise)
    ds.free()


@pytest.mark.parametrize("name", ["cornell", "one_weekend", "mixed_materials"])
def test_autotuned_layout_renders_the_same(cuda, name):
    spec, spp = _cases()[name]
    w, h = spec.width, spec.height
    sc = spec.to_scene()
    sc.build_bvh()
    fr = spec.camera.frame(w, h)
    a_ds = sc.upload()
    t_ds = sc.upload(layout="autotune", tune_depth=spec.depth)
    info = t_ds.layout
    assert info["kind"] in ("linear", "groups", "bvh") and info["probe_ms"] > 0
    a = render.render_accumulate(a_ds, fr, w, h, spp, spec.depth, background=spec.background, dof=spec.dof)
    b = render.render_accumulate(t_ds, fr, w, h, spp, spec.depth, background=spec.background, dof=spec.dof)
    # same sample streams; layouts can only differ on exact-t ties
    bad = (np.abs(a - b) > 1e-3 * (1 + np.abs(a)) * spp).any(axis=2)
    assert bad.mean() < 0.01
    # the decision is cached: a second upload reuses it without probing
    t2 = sc.upload(layout="autotune", tune_depth=spec.depth)
    assert t2.layout["kind"] == info["kind"] and t2.layout["leaf"] == info["leaf"]
    for d in (a_ds, t_ds, t2):
        d.free()


@pytest.mark.parametrize("name", ["cornell", "mixed_materials", "one_weekend", "small_icospheres"])
@pytest.mark.parametrize("nee", [False, True])
def test_wide_bvh_renders_the_same(cuda, name, nee):
    # the 4-wide copy holds the binary tree's own child boxes and leaves: the
    # same closest hits up to exact-t ties, so the same paths; primary hits
    # (exact-order traversal) stay on the binary tree and are identical
    spec, spp = _cases()[name]
    w, h = spec.width, spec.height
    sc = spec.to_scene()
    sc.build_bvh()
    fr = spec.camera.frame(w, h)
    b_ds = sc.upload(wide=False)
    w_ds = sc.upload()
    assert w_ds.nbytes > b_ds.nbytes
    np.testing.assert_array_equal(render.primary_hits(b_ds, fr, w, h), render.primary_hits(w_ds, fr, w, h))
    a, ca = render.render_accumulate(b_ds, fr, w, h, spp, spec.depth, background=spec.background, dof=spec.dof,
                                     nee=nee, counters=True)
    b, cb = render.render_accumulate(w_ds, fr, w, h, spp, spec.depth, background=spec.background, dof=spec.dof,
                                     nee=nee, counters=True)
    assert int(cb[2]) == 0  # no stack overflow on the wide tree
    bad = (np.abs(a - b) > 1e-3 * (1 + np.abs(a)) * spp).any(axis=2)
    assert bad.mean() < 0.01, bad.mean()
    np.testing.assert_allclose(a.mean((0, 1)), b.mean((0, 1)), rtol=1e-2, atol=1e-4)
    for d in (b_ds, w_ds):
        d.free()


@pytest.mark.parametrize("name", ["cornell", "mixed_materials", "one_weekend", "small_icospheres"])
@pytest.mark.parametrize("nee", [False, True])
def test_wavefront_engine_paired_with_per_pixel_kernel(cuda, name, nee):
    spec, spp = _cases()[name]
    w, h = spec.width, spec.height
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(w, h)
    a = render.render_accumulate(ds, fr, w, h, spp, spec.depth, background=spec.background, dof=spec.dof, nee=nee)
    # a small queue forces many regeneration/compaction rounds
    b, cnt = render.render_wavefront(ds, fr, w, h, spp, spec.depth, background=spec.background, dof=spec.dof,
                                     nee=nee, queue_capacity=4096, counters=True)
    assert int(cnt[1]) == w * h * spp  # every path accounted for exactly once
    bad = (np.abs(a - b) > 1e-3 * (1 + np.abs(a)) * spp).any(axis=2)
    assert bad.mean() < 0.01, bad.mean()
    np.testing.assert_allclose(a.mean((0, 1)), b.mean((0, 1)), rtol=1e-2, atol=1e-4)
    ds.free()


@pytest.mark.parametrize("name", ["cornell", "one_weekend"])
def test_grouped_layout_renders_the_same(cuda, name):
    # groups of the built tree's subtrees, primitives tested in the linear
    # scan's order: the same closest hits as the linear scan, so the same paths
    spec, _ = _cases()[name]
    w, h, spp = 48, 32, 8
    sc = spec.to_scene()
    sc.build_bvh()
    lin = sc.upload(layout="linear")
    fr = spec.camera.frame(w, h)
    a = render.render_accumulate(lin, fr, w, h, spp, spec.depth, background=spec.background, dof=spec.dof)
    for g in (1, 8, 16):
        grp = sc.upload(layout="groups", max_leaf=g)
        assert grp.layout["kind"] == "groups" and grp.layout["leaf"] == g
        b = render.render_accumulate(grp, fr, w, h, spp, spec.depth, background=spec.background, dof=spec.dof)
        bad = (np.abs(a - b) > 1e-3 * (1 + np.abs(a)) * spp).any(axis=2)
        assert bad.mean() < 0.005, (g, bad.mean())
        grp.free()
    lin.free()


def test_sample_slices_render_the_same(cuda):
    # a small frame splits its samples over several threads per pixel; the
    # samples (streams) are the same, only the FP32 summation grouping differs
    import ctypes as C

    from rayon_b200 import lib
    from rayon_b200._native import RenderOpts
    spec, _ = _cases()["one_weekend"]
    w, h, spp = 40, 24, 32
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(w, h)
    out = {}
    for slices in (1, 4, 5):
        o = RenderOpts()
        lib.rb_get_render_opts(C.byref(o))
        o.reserved[1] = slices
        lib.rb_set_render_opts(C.byref(o))
        out[slices], cnt = render.render_accumulate(ds, fr, w, h, spp, spec.depth, background=spec.background,
                                                    dof=spec.dof, counters=True)
        assert int(cnt[1]) == w * h * spp
        o.reserved[1] = 0
        lib.rb_set_render_opts(C.byref(o))
    for slices in (4, 5):
        np.testing.assert_allclose(out[slices], out[1], rtol=1e-4, atol=1e-4 * spp)
    ds.free()
