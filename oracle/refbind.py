"""Bindings to the reference-code drivers in oracle/_ref/ (test infrastructure).

librayon_ref_host.so: the reference's SceneDescription / buildBVH and its
RendererCPUParallel, driven through oracle/ref/ref_host_driver.cpp.
librayon_ref_cuda.so: the reference's CUDA renderer and a primary-hit probe,
driven through oracle/ref/ref_cuda_probe.cu (needs a GPU to run).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parent / "_ref"
HOST_LIB = REF_DIR / "librayon_ref_host.so"
CUDA_LIB = REF_DIR / "librayon_ref_cuda.so"

_host = None
_cuda = None

vp = C.c_void_p
dp = C.POINTER(C.c_double)


def host_available() -> bool:
    return HOST_LIB.exists()


def cuda_available() -> bool:
    return CUDA_LIB.exists()


def host():
    global _host
    if _host is None:
        from rayon_b200._native import MaterialDesc
        L = C.CDLL(str(HOST_LIB))
        L.refh_scene_create.restype = vp
        L.refh_scene_destroy.argtypes = [vp]
        L.refh_add_material.argtypes = [vp, C.POINTER(MaterialDesc)]
        L.refh_add_geoms.argtypes = [vp, C.POINTER(C.c_uint8), dp, C.POINTER(C.c_int32), C.c_int64]
        L.refh_build_bvh.argtypes = [vp]
        L.refh_num_nodes.argtypes = [vp]
        L.refh_num_nodes.restype = C.c_int64
        L.refh_root.argtypes = [vp]
        L.refh_export_bvh.argtypes = [vp, dp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_uint8),
                                      C.POINTER(C.c_uint8)]
        L.refh_export_order.argtypes = [vp, C.POINTER(C.c_int64)]
        L.refh_load_obj.argtypes = [vp, C.c_char_p, C.c_int, dp, dp]
        L.refh_load_obj.restype = C.c_int
        L.refh_num_geoms.argtypes = [vp]
        L.refh_num_geoms.restype = C.c_int64
        L.refh_export_triangles.argtypes = [vp, dp]
        L.refh_render_cpu_parallel.restype = C.c_double
        L.refh_render_cpu_parallel.argtypes = [vp, dp, dp, dp, C.c_double, C.c_int, C.c_int, C.c_int,
                                               C.POINTER(C.c_uint8), C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
        _host = L
    return _host


class RefScene:
    """A scene built through the reference's own SceneDescription."""

    def __init__(self, spec) -> None:
        L = host()
        self.L = L
        self.h = L.refh_scene_create()
        for m in spec.materials:
            L.refh_add_material(self.h, C.byref(m))
        kinds = np.ascontiguousarray(spec.kinds, np.uint8)
        params = np.ascontiguousarray(spec.params, np.float64)
        mats = np.ascontiguousarray(spec.mats, np.int32)
        L.refh_add_geoms(self.h, kinds.ctypes.data_as(C.POINTER(C.c_uint8)), params.ctypes.data_as(dp),
                         mats.ctypes.data_as(C.POINTER(C.c_int32)), int(kinds.shape[0]))
        self.n = int(kinds.shape[0])

    def build_bvh(self) -> None:
        self.L.refh_build_bvh(self.h)

    def export(self) -> dict:
        n = int(self.L.refh_num_nodes(self.h))
        bounds = np.zeros((n, 6), np.float64)
        a = np.zeros(n, np.int32)
        b = np.zeros(n, np.int32)
        leaf = np.zeros(n, np.uint8)
        ax = np.zeros(n, np.uint8)
        order = np.zeros(self.n, np.int64)
        self.L.refh_export_bvh(self.h, bounds.ctypes.data_as(dp), a.ctypes.data_as(C.POINTER(C.c_int32)),
                               b.ctypes.data_as(C.POINTER(C.c_int32)), leaf.ctypes.data_as(C.POINTER(C.c_uint8)),
                               ax.ctypes.data_as(C.POINTER(C.c_uint8)))
        self.L.refh_export_order(self.h, order.ctypes.data_as(C.POINTER(C.c_int64)))
        return dict(bounds=bounds, a=a, b=b, is_leaf=leaf, split_axis=ax, root=int(self.L.refh_root(self.h)),
                    order=order)

    def render_cpu_parallel(self, camera, width: int, height: int, spp: int):
        img = np.zeros(width * height * 3, np.uint8)
        th = C.c_int(0)
        rays = C.c_longlong(0)
        d3 = lambda v: (C.c_double * 3)(*[float(x) for x in v])  # noqa: E731
        secs = self.L.refh_render_cpu_parallel(self.h, d3(camera.look_from), d3(camera.look_at), d3(camera.vup),
                                               float(camera.vfov), int(width), int(height), int(spp),
                                               img.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(th), C.byref(rays))
        return secs, img.reshape(height, width, 3), th.value, rays.value

    def __del__(self) -> None:
        if getattr(self, "h", None):
            self.L.refh_scene_destroy(self.h)
            self.h = None


def reference_obj_triangles(path, mat: int, position=(0.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0)):
    """Loads an OBJ file with the reference's own OBJLoader::loadOBJ into a
    fresh reference SceneDescription; returns (count, n x 20 array: v0 v1 v2
    n0 n1 n2, has_normals, material) in insertion order."""
    import numpy as np
    L = host()
    sp = L.refh_scene_create()
    try:
        pos = (C.c_double * 3)(*position)
        sc = (C.c_double * 3)(*scale)
        n = L.refh_load_obj(sp, str(path).encode(), int(mat), pos, sc)
        g = int(L.refh_num_geoms(sp))
        out = np.zeros((g, 20), np.float64)
        L.refh_export_triangles(sp, out.ctypes.data_as(dp))
        return n, out
    finally:
        L.refh_scene_destroy(sp)
