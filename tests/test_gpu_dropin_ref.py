"""The drop-in display, heat-map and adaptive-sampling entry points against the
reference's own implementation of the same interface (renderer_cuda_device.cu
and shaders/render_acc_kernel.cu, built for sm_100a from its sources into
oracle/_ref/librayon_ref_cuda.so and loaded beside this library):

* convertAccumToDisplayCUDA (gammaCorrectKernel, render_acc_kernel.cu:11-44),
  renderSampleHeatmapCUDA (:50-115) and countConvergedPixels
  (renderer_cuda_device.cu:422-437) give the same bytes / count on the same
  device buffers;
* renderPixelsCUDAAccumulative with per-pixel sample counts
  (render_acc_kernel.cu:165-170, 241-271): on a scene whose every sample has
  the same radiance the accumulation and the count buffer are identical, call
  after call (the bookkeeping: skip when negative, the min_adaptive gate, the
  relative-luminance test, the sign flag); on the Cornell box, where the
  samples differ, the converged fraction and the displayed image agree with
  the reference's within the sampling scatter.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import refbind
from rayon_b200 import lib, render, scene as S, scenes

pytestmark = pytest.mark.gpu

u8p = C.POINTER(C.c_uint8)


@pytest.fixture(scope="module")
def ref(cuda):
    if not refbind.cuda_available():
        pytest.skip("oracle/_ref/librayon_ref_cuda.so not built")
    return refbind.cuda()


def _rand_accum(torch, n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    acc = torch.rand((n, 4), generator=g, device="cuda") * 40.0
    acc[::7] = 0.0
    acc[1::11] *= -1.0                     # negative sums clamp to 0
    acc[2::13] = 1e6                       # far above white
    return acc


@pytest.mark.parametrize("ch", [3, 4])
@pytest.mark.parametrize("with_counts", [False, True])
@pytest.mark.parametrize("gamma", [2.0, 2.2])
def test_display_bytes_match_reference(ref, cuda, ch, with_counts, gamma):
    torch = cuda
    w, h, spp = 173, 91, 24
    acc = _rand_accum(torch, w * h, 5)
    counts = None
    if with_counts:
        g = torch.Generator(device="cuda").manual_seed(6)
        cnt = torch.randint(-300, 301, (w * h,), generator=g, device="cuda", dtype=torch.int32)
        counts = C.c_void_p(cnt.data_ptr())
    ours = np.zeros(w * h * ch, np.uint8)
    theirs = np.ones(w * h * ch, np.uint8)
    lib.convertAccumToDisplayCUDA(C.c_void_p(acc.data_ptr()), ours.ctypes.data_as(u8p), w, h, ch, spp, gamma, counts)
    ref.convertAccumToDisplayCUDA(C.c_void_p(acc.data_ptr()), theirs.ctypes.data_as(u8p), w, h, ch, spp, gamma, counts)
    np.testing.assert_array_equal(ours, theirs)


@pytest.mark.parametrize("max_s", [0, 64, 1000])
@pytest.mark.parametrize("ch", [3, 4])
def test_heatmap_bytes_match_reference(ref, cuda, max_s, ch):
    torch = cuda
    w, h = 120, 77
    g = torch.Generator(device="cuda").manual_seed(max_s + ch)
    cnt = torch.randint(-1200, 1201, (w * h,), generator=g, device="cuda", dtype=torch.int32)
    ours = np.zeros(w * h * ch, np.uint8)
    theirs = np.ones(w * h * ch, np.uint8)
    lib.renderSampleHeatmapCUDA(C.c_void_p(cnt.data_ptr()), ours.ctypes.data_as(u8p), w, h, ch, max_s)
    ref.renderSampleHeatmapCUDA(C.c_void_p(cnt.data_ptr()), theirs.ctypes.data_as(u8p), w, h, ch, max_s)
    np.testing.assert_array_equal(ours, theirs)


def test_count_converged_and_buffer_helpers_match_reference(ref, cuda):
    torch = cuda
    n = 300_007
    g = torch.Generator(device="cuda").manual_seed(9)
    cnt = torch.randint(-50, 51, (n,), generator=g, device="cuda", dtype=torch.int32)
    assert lib.countConvergedPixels(C.c_void_p(cnt.data_ptr()), n) == \
        ref.countConvergedPixels(C.c_void_p(cnt.data_ptr()), n) == int((cnt < 0).sum())
    # allocate / reset / free through each library: a fresh buffer counts nothing
    for L in (lib, ref):
        p = C.c_void_p(None)
        L.allocateAdaptiveBuffer(C.byref(p), n)
        assert p.value
        assert L.countConvergedPixels(p, n) == 0
        L.resetAdaptiveBuffer(p, n)
        L.freeAdaptiveBuffer(p)
    assert lib.countConvergedPixels(None, n) == ref.countConvergedPixels(None, n) == 0


def _constant_scene():
    """One CONSTANT-material quad far larger than the view: every sample of
    every pixel returns exactly (0.5, 0.25, 0.125) (CONSTANT emits its colour
    and stops, cuda_raytracer.cuh:683-687), so the sums are exact in FP32."""
    B = scenes._Builder()
    m = B.mat(S.constant((0.5, 0.25, 0.125)))
    B.rect((-1000, -1000, -5), (2000, 0, 0), (0, 2000, 0), m)
    k, p, mm = B.arrays()
    return scenes.SceneSpec("constant", B.materials, k, p, mm, scenes.Camera((0, 0, 5), (0, 0, 0), (0, 1, 0), 40.0),
                            48, 32, 8, 4, background=0.0)


def _dropin_batch(L, scene_ptr, fr, w, h, add, total, depth, rng, dacc, host, counts, min_a, thr):
    return L.renderPixelsCUDAAccumulative(None, host.ctypes.data_as(C.POINTER(C.c_float)), scene_ptr, w, h,
                                          *[float(x) for x in fr[0:12]], add, total, depth, C.byref(rng),
                                          C.byref(dacc), *[float(x) for x in fr[12:18]], counts, min_a, thr)


def test_adaptive_dropin_bookkeeping_matches_reference(ref, cuda):
    torch = cuda
    spec = _constant_scene()
    w, h = spec.width, spec.height
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    rs = refbind.RefCudaScene(spec)
    fr = refbind.camera_frame(spec.camera, w, h)
    lib.setBackgroundIntensity(0.0)
    ref.setBackgroundIntensity(0.0)
    state = {}
    for name, L, sp in (("ours", lib, ds.handle), ("ref", ref, rs.device)):
        state[name] = dict(L=L, sp=sp, rng=C.c_void_p(None), acc=C.c_void_p(None),
                           host=np.zeros(w * h * 3, np.float32),
                           counts=torch.zeros(w * h, dtype=torch.int32, device="cuda"))
    # pre-converged pixels (negative counts) are skipped by both
    for st in state.values():
        st["counts"][::5] = -3
    total = 0
    for add in (8, 8, 8, 16):
        total += add
        for st in state.values():
            n = _dropin_batch(st["L"], st["sp"], fr, w, h, add, total, spec.depth, st["rng"], st["acc"], st["host"],
                              C.c_void_p(st["counts"].data_ptr()), 16, 0.01)
            assert n == w * h * add
        torch.cuda.synchronize()
        np.testing.assert_array_equal(state["ours"]["host"], state["ref"]["host"])
        np.testing.assert_array_equal(state["ours"]["counts"].cpu().numpy(), state["ref"]["counts"].cpu().numpy())
    c = state["ours"]["counts"].cpu().numpy()
    assert (c[::5] == -3).all() and (c[c != -3] == -16).all()   # converged at the min_adaptive gate
    # displayed with the per-pixel counts: same bytes
    imgs = []
    for st in state.values():
        out = np.zeros(w * h * 3, np.uint8)
        st["L"].convertAccumToDisplayCUDA(st["acc"], out.ctypes.data_as(u8p), w, h, 3, total, 2.0,
                                          C.c_void_p(st["counts"].data_ptr()))
        imgs.append(out)
        st["L"].freeDeviceRandomStates(st["rng"])
        st["L"].freeDeviceAccumBuffer(st["acc"])
    np.testing.assert_array_equal(imgs[0], imgs[1])
    lib.setBackgroundIntensity(1.0)
    ref.setBackgroundIntensity(1.0)
    rs.free()
    ds.free()


def test_adaptive_dropin_cornell_statistics_match_reference(ref, cuda):
    """Cornell box, 64 x 64, batches of 16 spp up to 256, min_adaptive 32,
    threshold 0.05. Converged fractions and the count-normalised images of the
    two renderers agree within the scatter between two runs of ours (different
    sample streams)."""
    torch = cuda
    spec = scenes.cornell(width=64, height=64)
    w, h = 64, 64
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    rs = refbind.RefCudaScene(spec)
    fr = refbind.camera_frame(spec.camera, w, h)

    def run(L, sp, seed=None):
        L.setBackgroundIntensity(0.0)
        rng, acc = C.c_void_p(None), C.c_void_p(None)
        host = np.zeros(w * h * 3, np.float32)
        counts = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        total = 0
        ctx = render.options(seed=seed) if seed is not None else None
        if ctx:
            ctx.__enter__()
        try:
            for _ in range(16):
                total += 16
                _dropin_batch(L, sp, fr, w, h, 16, total, spec.depth, rng, acc, host, C.c_void_p(counts.data_ptr()),
                              32, 0.05)
        finally:
            if ctx:
                ctx.__exit__(None, None, None)
        c = counts.cpu().numpy()
        img = host.reshape(h, w, 3) / np.maximum(np.abs(c), 1).reshape(h, w, 1)
        L.freeDeviceRandomStates(rng)
        L.freeDeviceAccumBuffer(acc)
        L.setBackgroundIntensity(1.0)
        return (c < 0).mean(), np.abs(c).mean(), img

    fa, sa, a = run(lib, ds.handle, seed=1)
    fb, sb, b = run(lib, ds.handle, seed=2)
    fr_, sr, r = run(ref, rs.device)
    rs.free()
    ds.free()
    spread = abs(fa - fb)
    assert abs(0.5 * (fa + fb) - fr_) < max(0.03, 3 * spread), (fa, fb, fr_)
    assert abs(0.5 * (sa + sb) - sr) < 0.05 * sr + 3 * abs(sa - sb), (sa, sb, sr)
    noise = np.sqrt(((a - b) ** 2).mean())
    err = np.sqrt(((0.5 * (a + b) - r) ** 2).mean())
    # the mean of two of ours against one of theirs: expected ratio ~ sqrt(3/4 / 2) = 0.61 of noise
    assert err < 1.0 * noise, (err, noise)
