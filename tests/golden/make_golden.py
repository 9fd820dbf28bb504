"""Generates the golden fixtures in tests/golden/ from the reference's own code
and from the FP64 oracle.

  python tests/golden/make_golden.py --bvh        (CPU; needs oracle/_ref/librayon_ref_host.so)
  python tests/golden/make_golden.py --sdf        (CPU; needs oracle/_ref/librayon_ref_host.so)
  python tests/golden/make_golden.py --gpu OUTDIR (GPU; needs oracle/_ref/librayon_ref_cuda.so)
  python tests/golden/make_golden.py --oracle     (CPU; needs oracle/_build/liboracle.so)

--bvh: for each BVH case, the scene is built through the reference's
SceneDescription (addSphere / addRectangle / addTriangle) and its buildBVH;
the node array and the leaf-order permutation are saved (bvh_<case>.npz).
--sdf: pixel-centre hits (object, distance) of the hard-union SDF case through
the reference's CPU scene and SDFShape::hit (sdf_hits_ref.npz).
--gpu: for each hit case, pixel-centre primary-hit ids and distances from the
reference's own hit_aabb / intersect_geometry on the GPU (hits_<case>.npz),
and reference CUDA renders (refimg_<case>.npz) for converged-image RMSE
checks, each through renderPixelsCUDAAccumulative with the reference's
setters for the case (background, depth of field). Cameras come from the
reference's CameraBase.
--oracle: the FP64 oracle's converged Cornell box at 64x64 (4096 spp, next-event
estimation, background 0, seed 777), the ground truth of the benchmark's
equal-RMSE comparison (oracle_cornell64.npz); and, per benchmark workload at
its full size, the oracle's mean radiance on a seeded pixel subset at high spp
(oracle_px_<case>.npz), the ground truth of the per-configuration error.
"""
from __future__ import annotations

import argparse
import ctypes as C
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

from cases import BVH_CASES, HIT_CASES, ORACLE_PX_CASES, REFIMG_CASES, sdf_pin  # noqa: E402

from oracle import refbind  # noqa: E402


def make_bvh(out: Path) -> None:
    for name, fn in BVH_CASES.items():
        spec = fn()
        r = refbind.RefScene(spec)
        r.build_bvh()
        e = r.export()
        np.savez_compressed(out / f"bvh_{name}.npz", **e)
        print(name, spec.n, "nodes", e["a"].shape[0])


def make_sdf(out: Path) -> None:
    spec = sdf_pin()
    w, h = spec.width, spec.height
    fr = refbind.camera_frame(spec.camera, w, h)
    ids, t, n = refbind.RefScene(spec).cpu_primary(fr, w, h)
    np.savez_compressed(out / "sdf_hits_ref.npz", ids=ids, t=t, normal=n.astype(np.float32), frame=fr, width=w,
                        height=h)
    print("sdf_hits_ref hit fraction", (ids >= 0).mean())


def make_gpu(out: Path) -> None:
    L = refbind.cuda()
    for name, (fn, w, h) in HIT_CASES.items():
        spec = fn()
        rs = refbind.RefCudaScene(spec)
        fr = np.ascontiguousarray(refbind.camera_frame(spec.camera, w, h), np.float64)
        ids = np.zeros(w * h, np.int32)
        t = np.zeros(w * h, np.float32)
        dis = L.refc_primary(rs.h, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)),
                             ids.ctypes.data_as(C.POINTER(C.c_int32)), t.ctypes.data_as(C.POINTER(C.c_float)))
        assert dis == 0, f"probe disagrees with hit_scene on {dis} rays ({name})"
        np.savez_compressed(out / f"hits_{name}.npz", ids=ids.reshape(h, w), t=t.reshape(h, w), width=w, height=h)
        print("hits", name, w, h, "hit fraction", (ids >= 0).mean())
        rs.free()
    for name, (fn, w, h, spp, depth) in REFIMG_CASES.items():
        spec = fn()
        t0 = time.time()
        rs = refbind.RefCudaScene(spec)
        build_s = time.time() - t0
        fr = np.ascontiguousarray(refbind.camera_frame(spec.camera, w, h), np.float64)
        dof = spec.dof or (0.1, 10.0)
        L.refc_set_globals(1.0, spec.background, 0.8, 1.5, int(spec.dof is not None), dof[0], dof[1])
        acc = np.zeros(w * h * 3, np.float32)
        secs = L.refc_render(rs.h, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)), spp, 5, depth,
                             acc.ctypes.data_as(C.POINTER(C.c_float)))
        img = acc.reshape(h, w, 3)
        if w * h > 64 * 64:  # larger images keep the mean in half precision (far below the noise)
            np.savez_compressed(out / f"refimg_{name}.npz", mean=(img / spp).astype(np.float16), spp=spp, depth=depth,
                                width=w, height=h, seconds=secs, build_seconds=build_s)
        else:
            np.savez_compressed(out / f"refimg_{name}.npz", sum=img, spp=spp, depth=depth, width=w, height=h,
                                seconds=secs)
        print("refimg", name, w, h, spp, "mean", img.reshape(-1, 3).mean(0) / spp, "secs", secs, "build", build_s)
        rs.free()
    L.refc_set_globals(1.0, 1.0, 0.8, 1.5, 0, 0.1, 10.0)


def make_oracle(out: Path, which=None) -> None:
    from oracle.oracle import Globals, OracleScene
    from rayon_b200 import scenes
    if which is None or "cornell64" in which:
        spec = scenes.cornell(width=64, height=64)
        sc = spec.to_scene()
        sc.build_bvh()
        fr = spec.camera.frame(64, 64)
        t0 = time.time()
        ref, _ = OracleScene(sc).render(fr, 64, 64, 4096, spec.depth, Globals(background=0.0, nee=True), seed=777)
        secs = time.time() - t0
        img = (ref.reshape(64, 64, 3) / 4096).astype(np.float32)
        np.savez_compressed(out / "oracle_cornell64.npz", mean=img, spp=4096, depth=spec.depth, seed=777,
                            seconds=secs)
        print("oracle_cornell64 mean", img.reshape(-1, 3).mean(0), "secs", secs)
    for name, (fn, npx, spp) in ORACLE_PX_CASES.items():
        if which is not None and name not in which:
            continue
        spec = fn()
        w, h = spec.width, spec.height
        sc = spec.to_scene()
        sc.build_bvh()
        fr = spec.camera.frame(w, h)
        px = np.sort(np.random.default_rng(2024).choice(w * h, size=npx, replace=False)).astype(np.int32)
        g = Globals(background=spec.background, dof=spec.dof is not None,
                    aperture=spec.dof[0] if spec.dof else 0.1, focus=spec.dof[1] if spec.dof else 10.0)
        o = OracleScene(sc, sdf=(spec.sdf_blend, spec.sdf_steps, spec.sdf_eps))
        t0 = time.time()
        s, cnt = o.render(fr, w, h, spp, spec.depth, g, seed=99991, pixels=px)
        secs = time.time() - t0
        np.savez_compressed(out / f"oracle_px_{name}.npz", pixels=px, mean=s / spp, spp=spp, width=w, height=h,
                            depth=spec.depth, seconds=secs, counters=cnt)
        print("oracle_px", name, npx, "px", spp, "spp", "secs", round(secs, 1), "mean", (s / spp).mean(0))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--bvh", action="store_true")
    ap.add_argument("--sdf", action="store_true")
    ap.add_argument("--gpu", default=None)
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("--only", nargs="*", default=None, help="--oracle: only these cases")
    a = ap.parse_args()
    if a.oracle:
        make_oracle(HERE, a.only)
    if a.bvh:
        make_bvh(HERE)
    if a.sdf:
        make_sdf(HERE)
    if a.gpu:
        o = Path(a.gpu)
        o.mkdir(parents=True, exist_ok=True)
        make_gpu(o)
