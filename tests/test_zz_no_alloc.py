"""convertAccumToDisplayNoAlloc: the allocation-free display conversion gives the
same image as convertAccumToDisplayCUDA, on two calls in a row that share its
fixed staging array, with and without per-pixel sample counts, for a strip
taller than a 2-D launch grid could cover; it leaves the device's free memory
unchanged and refuses images larger than that array.

It exists for callers that cannot allocate device memory when they want a
frame: device memory owned by another allocator or held to a fixed budget,
or loops that must avoid cudaMalloc's implicit device-wide synchronisation."""
import ctypes as C

import numpy as np
import pytest

from rayon_b200 import lib, scenes

pytestmark = pytest.mark.gpu

lib.convertAccumToDisplayNoAlloc.restype = C.c_int
lib.convertAccumToDisplayNoAlloc.argtypes = [C.c_void_p, C.POINTER(C.c_uint8), C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.c_float, C.c_void_p]


def _frame_accum(ds, spec, w, h, spp, rng, dacc):
    fr = spec.camera.frame(w, h)
    n = lib.renderPixelsCUDAAccumulative(None, None, ds.handle, w, h, *fr[0:12], spp, spp, spec.depth, C.byref(rng),
                                         C.byref(dacc), *fr[12:18], None, 32, 0.01)
    assert n == w * h * spp


def _existing(dacc, w, h, ch, spp, gamma=2.0, counts=None):
    out = np.zeros(w * h * ch, np.uint8)
    lib.convertAccumToDisplayCUDA(dacc, out.ctypes.data_as(C.POINTER(C.c_uint8)), w, h, ch, spp, gamma, counts)
    return out


def _noalloc(dacc, w, h, ch, spp, gamma=2.0, counts=None):
    out = np.full(w * h * ch, 7, np.uint8)
    st = lib.convertAccumToDisplayNoAlloc(dacc, out.ctypes.data_as(C.POINTER(C.c_uint8)), w, h, ch, spp, gamma,
                                          counts)
    assert st == 0, lib.rb_last_error()
    return out


def test_no_alloc_display_matches_existing(cuda):
    spec = scenes.cornell(width=160, height=120)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    lib.setBackgroundIntensity(0.0)
    # two calls in a row with different content and shapes share the array
    for (w, h, ch, spp) in [(160, 120, 3, 8), (96, 64, 4, 4)]:
        rng, dacc = C.c_void_p(None), C.c_void_p(None)
        _frame_accum(ds, spec, w, h, spp, rng, dacc)
        a = _existing(dacc, w, h, ch, spp)
        b = _noalloc(dacc, w, h, ch, spp)
        np.testing.assert_array_equal(a, b)
        lib.freeDeviceRandomStates(rng)
        lib.freeDeviceAccumBuffer(dacc)
    lib.setBackgroundIntensity(1.0)
    ds.free()


def test_no_alloc_counts_strip_and_free_memory(cuda):
    torch = cuda
    g = torch.Generator(device="cuda").manual_seed(3)
    # a 1 x 600,000 strip: more rows than a (32 x 8)-block 2-D grid can cover
    w, h, ch, spp = 1, 600_000, 3, 16
    acc = torch.rand((w * h, 4), generator=g, device="cuda") * 24.0
    # per-pixel counts: converged pixels hold negative counts, a few zeros
    counts = torch.randint(-64, 65, (w * h,), generator=g, device="cuda", dtype=torch.int32)
    a = _existing(C.c_void_p(acc.data_ptr()), w, h, ch, spp, counts=C.c_void_p(counts.data_ptr()))
    b = _noalloc(C.c_void_p(acc.data_ptr()), w, h, ch, spp, counts=C.c_void_p(counts.data_ptr()))
    np.testing.assert_array_equal(a, b)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in range(3):  # repeated calls allocate nothing
        b2 = _noalloc(C.c_void_p(acc.data_ptr()), w, h, ch, spp, counts=C.c_void_p(counts.data_ptr()))
        np.testing.assert_array_equal(a, b2)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_no_alloc_rejects_oversize(cuda):
    out = np.zeros(16, np.uint8)
    # 2048 x 1025 x 4 bytes is one row more than the 8 MiB staging array
    st = lib.convertAccumToDisplayNoAlloc(C.c_void_p(16), out.ctypes.data_as(C.POINTER(C.c_uint8)), 2048, 1025, 4, 1,
                                          2.0, None)
    assert st < 0
    assert "exceeds" in lib.rb_last_error().decode()
