"""RayON's unmodified offline CUDA renderer running on this library: the Cornell
box rendered by the reference's RendererCUDA::render
(gpu_renderers/renderer_cuda_host.hpp:23-74) through its RenderCoordinator,
with the scene built by its SceneDescription (and buildBVH), its camera from
CameraBase, its progress chunks and its host-side gamma conversion
(render_utils.hpp:41-74), every CUDA call resolving to librayon_b200.so
(oracle/_ref/librayon_dropin.so, built by oracle/ref/Makefile with
--no-undefined). The bytes it writes must match the reference renderer's own
image of the same frame (tests/golden/refimg_cornell.npz, 4096 spp, converted
by the same host function) within the sampling noise."""
import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from cases import REFIMG_CASES  # noqa: E402

from oracle.refbind import RefMaterial, as_ref_material  # noqa: E402
from rayon_b200 import lib, render  # noqa: E402

ROOT = Path(__file__).resolve().parent.parent
DROPIN = ROOT / "oracle" / "_ref" / "librayon_dropin.so"
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin(cuda):
    if not DROPIN.exists():
        pytest.skip("oracle/_ref/librayon_dropin.so not built")
    L = C.CDLL(str(DROPIN), mode=os.RTLD_NOW)
    dp = C.POINTER(C.c_double)
    L.dropin_render_offline.restype = C.c_longlong
    L.dropin_render_offline.argtypes = [C.POINTER(RefMaterial), C.c_int, C.POINTER(C.c_uint8), dp,
                                        C.POINTER(C.c_int32), C.c_int64, C.c_int, dp, dp, dp, C.c_double, C.c_int,
                                        C.c_int, C.c_int, C.c_float, C.POINTER(C.c_uint8)]
    L.dropin_accum_to_image.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_float,
                                        C.POINTER(C.c_uint8)]
    return L


def _render(L, spec, w, h, spp):
    mats = (RefMaterial * len(spec.materials))(*[as_ref_material(m) for m in spec.materials])
    k = np.ascontiguousarray(spec.kinds, np.uint8)
    p = np.ascontiguousarray(spec.params, np.float64)
    m = np.ascontiguousarray(spec.mats, np.int32)
    d3 = lambda v: (C.c_double * 3)(*[float(x) for x in v])  # noqa: E731
    out = np.zeros(w * h * 3, np.uint8)
    rays = L.dropin_render_offline(mats, len(spec.materials), k.ctypes.data_as(C.POINTER(C.c_uint8)),
                                   p.ctypes.data_as(C.POINTER(C.c_double)), m.ctypes.data_as(C.POINTER(C.c_int32)),
                                   k.shape[0], 1, d3(spec.camera.look_from), d3(spec.camera.look_at),
                                   d3(spec.camera.vup), float(spec.camera.vfov), w, h, spp, float(spec.background),
                                   out.ctypes.data_as(C.POINTER(C.c_uint8)))
    assert rays == w * h * spp, (rays, lib.rb_last_error())
    return out.reshape(h, w, 3).astype(np.float64)


def test_reference_renderer_on_this_library_matches_reference_image(dropin):
    fn, w, h, spp, depth = REFIMG_CASES["cornell"]
    assert depth == 16   # RendererCUDA renders at CameraBase::max_depth = 16
    spec = fn()
    g = np.load(Path(__file__).resolve().parent / "golden" / "refimg_cornell.npz")
    assert (int(g["width"]), int(g["height"]), int(g["spp"])) == (w, h, spp)
    ref = np.zeros(w * h * 3, np.uint8)
    acc = np.ascontiguousarray(g["sum"].reshape(-1), np.float32)
    dropin.dropin_accum_to_image(acc.ctypes.data_as(C.POINTER(C.c_float)), w, h, spp, 2.0,
                                 ref.ctypes.data_as(C.POINTER(C.c_uint8)))
    ref = ref.reshape(h, w, 3).astype(np.float64)
    with render.options(seed=11):
        a = _render(dropin, spec, w, h, spp)
    with render.options(seed=12):
        b = _render(dropin, spec, w, h, spp)
    noise = np.sqrt(((a - b) ** 2).mean())
    err = np.sqrt(((a - ref) ** 2).mean())
    assert a.mean() > 20           # a lit image, not a black frame
    assert err < 1.35 * noise + 0.5, (err, noise)
