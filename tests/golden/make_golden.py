"""Generates the golden fixtures in tests/golden/ from the reference's own code.

  python tests/golden/make_golden.py --bvh        (CPU; needs oracle/_ref/librayon_ref_host.so)
  python tests/golden/make_golden.py --gpu OUTDIR (GPU; needs oracle/_ref/librayon_ref_cuda.so)
  python tests/golden/make_golden.py --oracle     (CPU; needs oracle/_build/liboracle.so)

--bvh: for each BVH case, the scene is built through the reference's
SceneDescription (addSphere / addRectangle / addTriangle) and its buildBVH;
the node array and the leaf-order permutation are saved (bvh_<case>.npz).
--gpu: for each hit case, pixel-centre primary-hit ids and distances from the
reference's own hit_aabb / intersect_geometry on the GPU (hits_<case>.npz),
and reference CUDA renders of small scenes (refimg_<case>.npz) for RMSE checks.
--oracle: the FP64 oracle's converged Cornell box at 64x64 (4096 spp, next-event
estimation, background 0, seed 777), the ground truth of the benchmark's
equal-RMSE comparison (oracle_cornell64.npz).
"""
from __future__ import annotations

import argparse
import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

from cases import BVH_CASES, HIT_CASES  # noqa: E402

from oracle import refbind  # noqa: E402


def make_bvh(out: Path) -> None:
    for name, fn in BVH_CASES.items():
        spec = fn()
        r = refbind.RefScene(spec)
        r.build_bvh()
        e = r.export()
        np.savez_compressed(out / f"bvh_{name}.npz", **e)
        print(name, spec.n, "nodes", e["a"].shape[0])


def _cuda_lib():
    from rayon_b200._native import MaterialDesc
    L = C.CDLL(str(refbind.CUDA_LIB))
    L.refc_scene_create.restype = C.c_void_p
    L.refc_scene_create.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.c_double),
                                    C.POINTER(C.c_int32), C.c_int64, C.c_int]
    L.refc_scene_destroy.argtypes = [C.c_void_p]
    L.refc_primary.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int32),
                               C.POINTER(C.c_float)]
    L.refc_set_globals.argtypes = [C.c_float] * 4 + [C.c_int, C.c_float, C.c_float]
    L.refc_render.restype = C.c_double
    L.refc_render.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int,
                              C.POINTER(C.c_float)]
    L.refc_render_device.restype = C.c_float
    L.refc_render_device.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_int, C.c_int,
                                     C.POINTER(C.c_float)]
    return L, MaterialDesc


def ref_cuda_scene(L, MaterialDesc, spec):
    mats = (MaterialDesc * len(spec.materials))(*spec.materials)
    k = np.ascontiguousarray(spec.kinds, np.uint8)
    p = np.ascontiguousarray(spec.params, np.float64)
    m = np.ascontiguousarray(spec.mats, np.int32)
    h = L.refc_scene_create(C.cast(mats, C.c_void_p), len(spec.materials), C.sizeof(MaterialDesc),
                            k.ctypes.data_as(C.POINTER(C.c_uint8)), p.ctypes.data_as(C.POINTER(C.c_double)),
                            m.ctypes.data_as(C.POINTER(C.c_int32)), k.shape[0], 1)
    return h


def make_gpu(out: Path) -> None:
    L, MaterialDesc = _cuda_lib()
    for name, (fn, w, h) in HIT_CASES.items():
        spec = fn()
        sh = ref_cuda_scene(L, MaterialDesc, spec)
        fr = np.ascontiguousarray(spec.camera.frame(w, h), np.float64)
        ids = np.zeros(w * h, np.int32)
        t = np.zeros(w * h, np.float32)
        dis = L.refc_primary(sh, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)), ids.ctypes.data_as(C.POINTER(C.c_int32)),
                             t.ctypes.data_as(C.POINTER(C.c_float)))
        assert dis == 0, f"probe disagrees with hit_scene on {dis} rays ({name})"
        np.savez_compressed(out / f"hits_{name}.npz", ids=ids.reshape(h, w), t=t.reshape(h, w), width=w, height=h)
        print("hits", name, w, h, "hit fraction", (ids >= 0).mean())
        L.refc_scene_destroy(sh)
    # reference CUDA images for RMSE checks (small, converged-ish)
    for name, fn, w, h, spp, depth in [("cornell", HIT_CASES["cornell"][0], 64, 64, 4096, 16),
                                       ("mixed_materials", HIT_CASES["mixed_materials"][0], 48, 36, 4096, 8)]:
        spec = fn()
        sh = ref_cuda_scene(L, MaterialDesc, spec)
        fr = np.ascontiguousarray(spec.camera.frame(w, h), np.float64)
        dof = spec.dof or (0.1, 10.0)
        L.refc_set_globals(1.0, spec.background, 0.8, 1.5, int(spec.dof is not None), dof[0], dof[1])
        acc = np.zeros(w * h * 3, np.float32)
        secs = L.refc_render(sh, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)), spp, 5, depth,
                             acc.ctypes.data_as(C.POINTER(C.c_float)))
        np.savez_compressed(out / f"refimg_{name}.npz", sum=acc.reshape(h, w, 3), spp=spp, depth=depth, width=w,
                            height=h, seconds=secs)
        print("refimg", name, w, h, spp, "mean", acc.reshape(-1, 3).mean(0) / spp, "secs", secs)
        L.refc_scene_destroy(sh)


def make_oracle(out: Path) -> None:
    import time

    from oracle.oracle import Globals, OracleScene
    from rayon_b200 import scenes
    spec = scenes.cornell(width=64, height=64)
    sc = spec.to_scene()
    sc.build_bvh()
    fr = spec.camera.frame(64, 64)
    t0 = time.time()
    ref, _ = OracleScene(sc).render(fr, 64, 64, 4096, spec.depth, Globals(background=0.0, nee=True), seed=777)
    secs = time.time() - t0
    img = (ref.reshape(64, 64, 3) / 4096).astype(np.float32)
    np.savez_compressed(out / "oracle_cornell64.npz", mean=img, spp=4096, depth=spec.depth, seed=777, seconds=secs)
    print("oracle_cornell64 mean", img.reshape(-1, 3).mean(0), "secs", secs)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--bvh", action="store_true")
    ap.add_argument("--gpu", default=None)
    ap.add_argument("--oracle", action="store_true")
    a = ap.parse_args()
    if a.oracle:
        make_oracle(HERE)
    if a.bvh:
        make_bvh(HERE)
    if a.gpu:
        o = Path(a.gpu)
        o.mkdir(parents=True, exist_ok=True)
        make_gpu(o)
