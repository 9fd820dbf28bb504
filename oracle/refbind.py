"""Bindings to the reference-code drivers in oracle/_ref/ (test infrastructure).

librayon_ref_host.so: the reference's SceneDescription / buildBVH, its
CameraBase frame, its CPU scene's primary hits and its RendererCPUParallel,
driven through oracle/ref/ref_host_driver.cpp.
librayon_ref_cuda.so: the reference's CUDA renderer (its whole extern "C"
interface, renderer_cuda_device.cuh:8-67) and a primary-hit probe, driven
through oracle/ref/ref_cuda_probe.cu (needs a GPU to run).

Nothing here imports the rayon_b200 package, so a process that only drives
the reference (bench.py --impl reference) never loads this project's library.
Scenes come in as SceneSpec-like objects: `materials` (ctypes structures with
the layout of rb_material_desc, include/rayon_b200_scene.h), `kinds`,
`params`, `mats` arrays, and a camera with look_from / look_at / vup / vfov.
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
fp = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)
u8p = C.POINTER(C.c_uint8)


class RefMaterial(C.Structure):
    """The oracle's own mirror of rb_material_desc (include/rayon_b200_scene.h),
    the plain-data form of the reference's Scene::MaterialDesc
    (scene_description.hpp:58-101) that the drivers convert field by field."""
    _fields_ = [
        ("type", C.c_int32),
        ("albedo", C.c_double * 3),
        ("emission", C.c_double * 3),
        ("roughness", C.c_float), ("metallic", C.c_float), ("refractive_index", C.c_float),
        ("transmission", C.c_float), ("anisotropy", C.c_float),
        ("eta", C.c_double * 3),
        ("k", C.c_double * 3),
        ("texture_id", C.c_int32),
        ("film_thickness", C.c_float), ("film_ior", C.c_float),
        ("pattern", C.c_int32),
        ("pattern_color", C.c_double * 3),
        ("pattern_param1", C.c_float), ("pattern_param2", C.c_float),
    ]


def as_ref_material(m) -> RefMaterial:
    """A material as RefMaterial: RefMaterial itself, any ctypes structure of
    the same layout (copied byte for byte), or a dict of field values (the
    MaterialDesc() defaults for the rest: albedo 0.7, texture -1, film 400 nm
    at IOR 1.33, refractive index 1)."""
    if isinstance(m, RefMaterial):
        return m
    if isinstance(m, C.Structure):
        if C.sizeof(m) != C.sizeof(RefMaterial):
            raise TypeError("material structure does not have the rb_material_desc layout")
        return RefMaterial.from_buffer_copy(m)
    r = RefMaterial()
    r.albedo[:] = [0.7, 0.7, 0.7]
    r.refractive_index, r.texture_id, r.film_thickness, r.film_ior = 1.0, -1, 400.0, 1.33
    for k, v in dict(m).items():
        if isinstance(getattr(r, k), C.Array):
            getattr(r, k)[:] = [float(x) for x in v]
        else:
            setattr(r, k, v)
    return r


def host_available() -> bool:
    return HOST_LIB.exists()


def cuda_available() -> bool:
    return CUDA_LIB.exists()


def host():
    global _host
    if _host is None:
        L = C.CDLL(str(HOST_LIB))
        L.refh_scene_create.restype = vp
        L.refh_scene_destroy.argtypes = [vp]
        L.refh_add_material.argtypes = [vp, C.POINTER(RefMaterial)]
        L.refh_add_geoms.argtypes = [vp, u8p, dp, i32p, C.c_int64]
        L.refh_build_bvh.argtypes = [vp]
        L.refh_num_nodes.argtypes = [vp]
        L.refh_num_nodes.restype = C.c_int64
        L.refh_root.argtypes = [vp]
        L.refh_export_bvh.argtypes = [vp, dp, i32p, i32p, u8p, u8p]
        L.refh_export_order.argtypes = [vp, C.POINTER(C.c_int64)]
        L.refh_load_obj.argtypes = [vp, C.c_char_p, C.c_int, dp, dp]
        L.refh_load_obj.restype = C.c_int
        L.refh_num_geoms.argtypes = [vp]
        L.refh_num_geoms.restype = C.c_int64
        L.refh_export_triangles.argtypes = [vp, dp]
        L.refh_render_cpu_parallel.restype = C.c_double
        L.refh_render_cpu_parallel.argtypes = [vp, dp, dp, dp, C.c_double, C.c_int, C.c_int, C.c_int, u8p,
                                               C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
        L.refh_camera_frame.argtypes = [dp, dp, dp, C.c_double, C.c_int, C.c_int, dp]
        L.refh_cpu_primary.restype = C.c_int64
        L.refh_cpu_primary.argtypes = [vp, C.c_int, C.c_int, dp, i32p, dp, dp]
        _host = L
    return _host


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def camera_frame(camera, width: int, height: int) -> np.ndarray:
    """The reference's own frame (CameraBase::buildFrame after updateFrame,
    camera_base.hpp:47-99) for a camera with look_from / look_at / vup / vfov:
    center, pixel00, delta_u, delta_v, u, v, w as 21 doubles."""
    out = np.zeros(21, np.float64)
    host().refh_camera_frame(_d3(camera.look_from), _d3(camera.look_at), _d3(camera.vup), float(camera.vfov),
                             int(width), int(height), out.ctypes.data_as(dp))
    return out


class RefScene:
    """A scene built through the reference's own SceneDescription."""

    def __init__(self, spec) -> None:
        L = host()
        self.L = L
        self.h = L.refh_scene_create()
        for m in spec.materials:
            L.refh_add_material(self.h, C.byref(as_ref_material(m)))
        kinds = np.ascontiguousarray(spec.kinds, np.uint8)
        params = np.ascontiguousarray(spec.params, np.float64)
        mats = np.ascontiguousarray(spec.mats, np.int32)
        L.refh_add_geoms(self.h, kinds.ctypes.data_as(u8p), params.ctypes.data_as(dp), mats.ctypes.data_as(i32p),
                         int(kinds.shape[0]))
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
        self.L.refh_export_bvh(self.h, bounds.ctypes.data_as(dp), a.ctypes.data_as(i32p), b.ctypes.data_as(i32p),
                               leaf.ctypes.data_as(u8p), ax.ctypes.data_as(u8p))
        self.L.refh_export_order(self.h, order.ctypes.data_as(C.POINTER(C.c_int64)))
        return dict(bounds=bounds, a=a, b=b, is_leaf=leaf, split_axis=ax, root=int(self.L.refh_root(self.h)),
                    order=order)

    def cpu_primary(self, frame, width: int, height: int):
        """Pixel-centre closest hits through the reference's CPU scene (unit
        ray directions): object index (insertion order) or -1, distance t,
        normal (as recorded by the shape's hit)."""
        fr = np.ascontiguousarray(frame, np.float64)
        ids = np.zeros(width * height, np.int32)
        t = np.zeros(width * height, np.float64)
        n = np.zeros((width * height, 3), np.float64)
        self.L.refh_cpu_primary(self.h, int(width), int(height), fr.ctypes.data_as(dp), ids.ctypes.data_as(i32p),
                                t.ctypes.data_as(dp), n.ctypes.data_as(dp))
        return ids.reshape(height, width), t.reshape(height, width), n.reshape(height, width, 3)

    def render_cpu_parallel(self, camera, width: int, height: int, spp: int):
        img = np.zeros(width * height * 3, np.uint8)
        th = C.c_int(0)
        rays = C.c_longlong(0)
        secs = self.L.refh_render_cpu_parallel(self.h, _d3(camera.look_from), _d3(camera.look_at), _d3(camera.vup),
                                               float(camera.vfov), int(width), int(height), int(spp),
                                               img.ctypes.data_as(u8p), C.byref(th), C.byref(rays))
        return secs, img.reshape(height, width, 3), th.value, rays.value

    def __del__(self) -> None:
        if getattr(self, "h", None):
            self.L.refh_scene_destroy(self.h)
            self.h = None


def reference_obj_triangles(path, mat: int, position=(0.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0)):
    """Loads an OBJ file with the reference's own OBJLoader::loadOBJ into a
    fresh reference SceneDescription; returns (count, n x 20 array: v0 v1 v2
    n0 n1 n2, has_normals, material) in insertion order."""
    L = host()
    sp = L.refh_scene_create()
    try:
        n = L.refh_load_obj(sp, str(path).encode(), int(mat), _d3(position), _d3(scale))
        g = int(L.refh_num_geoms(sp))
        out = np.zeros((g, 20), np.float64)
        L.refh_export_triangles(sp, out.ctypes.data_as(dp))
        return n, out
    finally:
        L.refh_scene_destroy(sp)


# ---------------------------------------------------------------------------
# The reference's CUDA renderer (GPU)


def cuda():
    """librayon_ref_cuda.so with the probe driver's refc_* entry points and the
    reference's own extern "C" renderer interface (renderer_cuda_device.cuh)."""
    global _cuda
    if _cuda is None:
        L = C.CDLL(str(CUDA_LIB))
        L.refc_scene_create.restype = vp
        L.refc_scene_create.argtypes = [vp, C.c_int, C.c_int, u8p, dp, i32p, C.c_int64, C.c_int]
        L.refc_scene_destroy.argtypes = [vp]
        L.refc_scene_device.restype = vp
        L.refc_scene_device.argtypes = [vp]
        L.refc_primary.argtypes = [vp, C.c_int, C.c_int, dp, i32p, fp]
        L.refc_set_globals.argtypes = [C.c_float] * 4 + [C.c_int, C.c_float, C.c_float]
        L.refc_render.restype = C.c_double
        L.refc_render.argtypes = [vp, C.c_int, C.c_int, dp, C.c_int, C.c_int, C.c_int, fp]
        L.refc_render_device.restype = C.c_float
        L.refc_render_device.argtypes = [vp, C.c_int, C.c_int, dp, C.c_int, C.c_int, fp]
        # the reference's own interface
        L.renderPixelsCUDAAccumulative.restype = C.c_ulonglong
        L.renderPixelsCUDAAccumulative.argtypes = ([vp, fp, vp, C.c_int, C.c_int] + [C.c_double] * 12 +
                                                   [C.c_int, C.c_int, C.c_int, C.POINTER(vp), C.POINTER(vp)] +
                                                   [C.c_double] * 6 + [vp, C.c_int, C.c_float])
        L.convertAccumToDisplayCUDA.argtypes = [vp, u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, vp]
        L.renderSampleHeatmapCUDA.argtypes = [vp, u8p, C.c_int, C.c_int, C.c_int, C.c_int]
        L.countConvergedPixels.restype = C.c_int
        L.countConvergedPixels.argtypes = [vp, C.c_int]
        L.allocateAdaptiveBuffer.argtypes = [C.POINTER(vp), C.c_int]
        L.freeAdaptiveBuffer.argtypes = [vp]
        L.freeDeviceRandomStates.argtypes = [vp]
        L.freeDeviceAccumBuffer.argtypes = [vp]
        L.setBackgroundIntensity.argtypes = [C.c_float]
        L.setLightIntensity.argtypes = [C.c_float]
        L.setMetalFuzziness.argtypes = [C.c_float]
        L.setGlassRefractionIndex.argtypes = [C.c_float]
        L.setDOFEnabled.argtypes = [C.c_bool]
        L.setDOFAperture.argtypes = [C.c_float]
        L.setDOFFocusDistance.argtypes = [C.c_float]
        _cuda = L
    return _cuda


class RefCudaScene:
    """A scene built through the reference's SceneDescription (and its
    buildBVH) and uploaded by its CudaSceneBuilder::buildGPUScene."""

    def __init__(self, spec, build_bvh: bool = True) -> None:
        L = cuda()
        self.L = L
        mats = (RefMaterial * len(spec.materials))(*[as_ref_material(m) for m in spec.materials])
        k = np.ascontiguousarray(spec.kinds, np.uint8)
        p = np.ascontiguousarray(spec.params, np.float64)
        m = np.ascontiguousarray(spec.mats, np.int32)
        self.h = L.refc_scene_create(C.cast(mats, vp), len(spec.materials), C.sizeof(RefMaterial),
                                     k.ctypes.data_as(u8p), p.ctypes.data_as(dp), m.ctypes.data_as(i32p),
                                     int(k.shape[0]), int(build_bvh))
        if not self.h:
            raise RuntimeError("refc_scene_create failed")

    @property
    def device(self):
        """The reference's CudaScene::Scene* (a device pointer)."""
        return self.L.refc_scene_device(self.h)

    def free(self) -> None:
        if getattr(self, "h", None):
            self.L.refc_scene_destroy(self.h)
            self.h = None

    def __del__(self) -> None:
        try:
            self.free()
        except Exception:
            pass
