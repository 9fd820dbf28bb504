"""The per-pixel kernel's two schedules render the same sums bit for bit.

Grid mode launches one thread per pixel over a 2-D grid (sample slices on
grid z); fetch mode launches a persistent grid whose warps take 8 x 4-pixel
tiles of a sample slice from a counter. Each pixel's slice is computed by one
thread in sample order either way, so the FP32 sums, their Kahan terms and the
segment and path counters agree exactly, for frames whose width and height are
not multiples of the tile, for small frames that split their samples into
slices, with next-event estimation and with adaptive sample counts."""
import ctypes as C

import numpy as np
import pytest

from rayon_b200 import lib, render, scenes

pytestmark = pytest.mark.gpu


def _frame(torch, ds, spec, w, h, spp, schedule, counts=None, nee=False):
    fr = np.ascontiguousarray(spec.camera.frame(w, h), np.float64)
    buf = torch.zeros((2, w * h, 4), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(4, dtype=torch.int64, device="cuda")
    render.set_globals(background=spec.background, dof=spec.dof)
    with render.options(schedule=schedule, nee=nee):
        st = lib.rb_render_accumulate(ds.handle, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)), spp, 0, spec.depth,
                                      C.c_void_p(buf[0].data_ptr()), C.c_void_p(buf[1].data_ptr()),
                                      C.c_void_p(cnt.data_ptr()), None)
    assert st == 0, lib.rb_last_error()
    torch.cuda.synchronize()
    render.set_globals()
    return buf.cpu().numpy(), cnt.cpu().numpy()


@pytest.mark.parametrize("name,w,h,spp", [("cornell", 203, 117, 24), ("cornell", 640, 480, 8),
                                          ("one_weekend", 130, 75, 16), ("icospheres8", 97, 61, 8)])
@pytest.mark.parametrize("nee", [False, True])
def test_fetch_schedule_matches_grid(cuda, name, w, h, spp, nee):
    torch = cuda
    if name == "icospheres8":
        spec = scenes.icospheres(count=8, level=4)
    else:
        spec = getattr(scenes, name)()
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    a, ca = _frame(torch, ds, spec, w, h, spp, "grid", nee=nee)
    b, cb = _frame(torch, ds, spec, w, h, spp, "fetch", nee=nee)
    ds.free()
    assert a[0, :, :3].sum() > 0
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(ca[:3], cb[:3])
    assert ca[1] == w * h * spp


def test_fetch_schedule_adaptive_counts_match_grid(cuda):
    """Adaptive sampling through the drop-in renderPixelsCUDAAccumulative with
    per-pixel counts (some pixels converged before the first batch): the sums
    and the counts agree batch after batch."""
    torch = cuda
    spec = scenes.cornell(width=96, height=72)
    w, h = 96, 72
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    fr = spec.camera.frame(w, h)
    out = {}
    for schedule in ("grid", "fetch"):
        rng, dacc = C.c_void_p(None), C.c_void_p(None)
        host = np.zeros(w * h * 3, np.float32)
        counts = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        counts[::9] = -5          # converged before the first batch: skipped
        total = 0
        with render.options(schedule=schedule, seed=5):
            for add in (16, 16, 16):
                total += add
                n = lib.renderPixelsCUDAAccumulative(None, host.ctypes.data_as(C.POINTER(C.c_float)), ds.handle, w, h,
                                                     *[float(x) for x in fr[0:12]], add, total, spec.depth,
                                                     C.byref(rng), C.byref(dacc), *[float(x) for x in fr[12:18]],
                                                     C.c_void_p(counts.data_ptr()), 16, 0.05)
                assert n == w * h * add, lib.rb_last_error()
        torch.cuda.synchronize()
        out[schedule] = (host.copy(), counts.cpu().numpy())
        lib.freeDeviceRandomStates(rng)
        lib.freeDeviceAccumBuffer(dacc)
    ds.free()
    assert (out["grid"][1] < 0).any()
    np.testing.assert_array_equal(out["grid"][0], out["fetch"][0])
    np.testing.assert_array_equal(out["grid"][1], out["fetch"][1])
