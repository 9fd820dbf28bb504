"""convertAccumToDisplayNoAlloc: the allocation-free display conversion gives the
same image as convertAccumToDisplayCUDA, on two calls in a row that share its
fixed staging array, and refuses images larger than that array.

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


def _existing(dacc, w, h, ch, spp, gamma=2.0):
    out = np.zeros(w * h * ch, np.uint8)
    lib.convertAccumToDisplayCUDA(dacc, out.ctypes.data_as(C.POINTER(C.c_uint8)), w, h, ch, spp, gamma, None)
    return out


def _noalloc(dacc, w, h, ch, spp, gamma=2.0):
    out = np.full(w * h * ch, 7, np.uint8)
    st = lib.convertAccumToDisplayNoAlloc(dacc, out.ctypes.data_as(C.POINTER(C.c_uint8)), w, h, ch, spp, gamma, None)
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


def test_no_alloc_rejects_oversize(cuda):
    out = np.zeros(16, np.uint8)
    # 2048 x 1025 x 4 bytes is one row more than the 8 MiB staging array
    st = lib.convertAccumToDisplayNoAlloc(C.c_void_p(16), out.ctypes.data_as(C.POINTER(C.c_uint8)), 2048, 1025, 4, 1,
                                          2.0, None)
    assert st < 0
    assert "exceeds" in lib.rb_last_error().decode()
