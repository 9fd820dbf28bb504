"""Python mirror of the reference's scene-building API, over the C-ABI.

SceneDescription follows Scene::SceneDescription's builder interface
(src/rayon/scenes/scene_description.hpp:487-711) and its BVH build
(:717-925); the work is done in the native library. Material factories follow
MaterialDesc's (scene_description.hpp:104-245).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._native import MaterialDesc, UploadOpts, c_double_p, c_float_p, c_int32_p, c_int64_p, c_uint8_p, check, lib

# Scene::MaterialType numbering (scene_description.hpp:29-43)
LAMBERTIAN, METAL, MIRROR, ROUGH_MIRROR, GLASS, DIELECTRIC, LIGHT, CONSTANT, SHOW_NORMALS, SDF_MATERIAL, \
    ANISOTROPIC_METAL, THIN_FILM, CLEAR_COAT = range(13)
# Scene::GeometryType numbering (scene_description.hpp:252-260)
G_SPHERE, G_RECTANGLE, G_CUBE, G_DISPLACED_SPHERE, G_TRIANGLE, G_TRIANGLE_MESH, G_SDF = range(7)
# Scene::SDFType numbering (scene_description.hpp:296-309) + rounded box
SDF_SPHERE, SDF_BOX, SDF_TORUS, SDF_CAPSULE = 0, 1, 2, 3
SDF_ROUND_BOX = 32


def _d3(v) -> C.Array:
    a = (C.c_double * 3)(*[float(x) for x in v])
    return a


def material(type: int = LAMBERTIAN, albedo=(0.7, 0.7, 0.7), emission=(0, 0, 0), roughness=0.0, metallic=0.0,
             refractive_index=1.0, transmission=0.0, anisotropy=0.0, eta=(0, 0, 0), k=(0, 0, 0),
             film_thickness=400.0, film_ior=1.33, pattern=0, pattern_color=(0, 0, 0), pattern_param1=0.0,
             pattern_param2=0.0) -> MaterialDesc:
    m = MaterialDesc()
    lib.rb_material_default(C.byref(m))
    m.type = type
    m.albedo[:] = [float(x) for x in albedo]
    m.emission[:] = [float(x) for x in emission]
    m.roughness, m.metallic, m.refractive_index = roughness, metallic, refractive_index
    m.transmission, m.anisotropy = transmission, anisotropy
    m.eta[:] = [float(x) for x in eta]
    m.k[:] = [float(x) for x in k]
    m.film_thickness, m.film_ior = film_thickness, film_ior
    m.pattern = pattern
    m.pattern_color[:] = [float(x) for x in pattern_color]
    m.pattern_param1, m.pattern_param2 = pattern_param1, pattern_param2
    return m


def lambertian(color) -> MaterialDesc:
    return material(LAMBERTIAN, albedo=color)


def metal(color, roughness=0.0) -> MaterialDesc:
    return material(METAL, albedo=color, roughness=roughness, metallic=1.0)


def mirror(color) -> MaterialDesc:
    return material(MIRROR, albedo=color, metallic=1.0)


def glass(ior) -> MaterialDesc:
    return material(GLASS, albedo=(1, 1, 1), refractive_index=ior, transmission=1.0)


def light(emission) -> MaterialDesc:
    return material(LIGHT, albedo=(1, 1, 1), emission=emission)


def constant(color) -> MaterialDesc:
    return material(CONSTANT, albedo=color)


def anisotropic_metal(roughness, anisotropy, eta, k) -> MaterialDesc:
    return material(ANISOTROPIC_METAL, albedo=(1, 1, 1), roughness=roughness, anisotropy=anisotropy, metallic=1.0,
                    eta=eta, k=k)


def ggx_from_f0(roughness: float, f0: float) -> MaterialDesc:
    """GGX conductor with normal-incidence reflectance F0: k = 0, eta = (1 + sqrt F0) / (1 - sqrt F0)."""
    s = np.sqrt(f0)
    eta = (1 + s) / (1 - s)
    return anisotropic_metal(roughness, 0.0, (eta, eta, eta), (0.0, 0.0, 0.0))


def thin_film(thickness, film_ior=1.33, base_ior=1.0) -> MaterialDesc:
    return material(THIN_FILM, albedo=(1, 1, 1), film_thickness=thickness, film_ior=film_ior,
                    refractive_index=base_ior, transmission=1.0)


def clear_coat(color, coat_roughness=0.05, coat_ior=1.5) -> MaterialDesc:
    return material(CLEAR_COAT, albedo=color, roughness=coat_roughness, refractive_index=coat_ior)


@dataclass
class BVHExport:
    bounds: np.ndarray     # (n, 6) float64
    a: np.ndarray          # (n,) int32 left child / first geometry
    b: np.ndarray          # (n,) int32 right child / count
    is_leaf: np.ndarray    # (n,) uint8
    split_axis: np.ndarray  # (n,) uint8
    root: int


class SceneDescription:
    """Host scene (FP64) with the reference's builder interface."""

    def __init__(self) -> None:
        self._h = lib.rb_scene_create()
        if not self._h:
            raise RuntimeError("rb_scene_create failed")

    def __del__(self) -> None:
        h = getattr(self, "_h", None)
        if h and lib is not None:
            lib.rb_scene_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    # --- builder -------------------------------------------------------------
    def add_material(self, m: MaterialDesc) -> int:
        return check(lib.rb_scene_add_material(self._h, C.byref(m)), "add_material")

    def add_sphere(self, center, radius, mat_id) -> int:
        return check(lib.rb_scene_add_sphere(self._h, _d3(center), float(radius), int(mat_id)), "add_sphere")

    def add_displaced_sphere(self, center, radius, mat_id, displacement_scale=0.2, pattern_type=0) -> int:
        return check(lib.rb_scene_add_displaced_sphere(self._h, _d3(center), float(radius), int(mat_id),
                                                       float(displacement_scale), int(pattern_type)))

    def add_rectangle(self, corner, u, v, mat_id) -> int:
        return check(lib.rb_scene_add_rectangle(self._h, _d3(corner), _d3(u), _d3(v), int(mat_id)), "add_rectangle")

    def add_triangle(self, v0, v1, v2, mat_id) -> int:
        return check(lib.rb_scene_add_triangle(self._h, _d3(v0), _d3(v1), _d3(v2), int(mat_id)), "add_triangle")

    def add_triangle_with_normals(self, v0, v1, v2, n0, n1, n2, mat_id) -> int:
        return check(lib.rb_scene_add_triangle_with_normals(self._h, _d3(v0), _d3(v1), _d3(v2), _d3(n0), _d3(n1),
                                                            _d3(n2), int(mat_id)))

    def add_sdf(self, sdf_type, position, params, mat_id, rotation=(0, 0, 0)) -> int:
        return check(lib.rb_scene_add_sdf(self._h, int(sdf_type), _d3(position), _d3(params), _d3(rotation),
                                          int(mat_id)), "add_sdf")

    def add_spheres(self, cr: np.ndarray, mat_ids=None, mat_id: int = 0) -> int:
        cr = np.ascontiguousarray(cr, dtype=np.float64).reshape(-1, 4)
        mids = None if mat_ids is None else np.ascontiguousarray(mat_ids, dtype=np.int32)
        return check(lib.rb_scene_add_spheres(self._h, cr.ctypes.data_as(c_double_p),
                                              None if mids is None else mids.ctypes.data_as(c_int32_p),
                                              int(mat_id), cr.shape[0]), "add_spheres")

    def add_triangles(self, v: np.ndarray, mat_ids=None, mat_id: int = 0, normals=None) -> int:
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 9)
        nrm = None if normals is None else np.ascontiguousarray(normals, dtype=np.float64).reshape(-1, 9)
        mids = None if mat_ids is None else np.ascontiguousarray(mat_ids, dtype=np.int32)
        return check(lib.rb_scene_add_triangles(self._h, v.ctypes.data_as(c_double_p),
                                                None if nrm is None else nrm.ctypes.data_as(c_double_p),
                                                None if mids is None else mids.ctypes.data_as(c_int32_p),
                                                int(mat_id), v.shape[0]), "add_triangles")

    def load_obj(self, path, mat_id: int, position=(0.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0)) -> int:
        """Triangles of a Wavefront OBJ file (OBJLoader::loadOBJ semantics); returns their count."""
        return check(lib.rb_scene_load_obj(self._h, str(path).encode(), int(mat_id), _d3(position), _d3(scale)),
                     "load_obj")

    def set_visible(self, geom_index: int, visible: bool) -> None:
        check(lib.rb_scene_set_visible(self._h, int(geom_index), int(bool(visible))), "set_visible")

    def set_sdf_blend(self, k: float, max_steps: int = 256, epsilon: float = 1e-4) -> None:
        check(lib.rb_scene_set_sdf_blend(self._h, float(k), int(max_steps), float(epsilon)), "set_sdf_blend")

    @property
    def num_geometries(self) -> int:
        return int(lib.rb_scene_num_geometries(self._h))

    @property
    def num_materials(self) -> int:
        return int(lib.rb_scene_num_materials(self._h))

    # --- BVH -------------------------------------------------------------------
    def build_bvh(self, max_leaf: int = 4, threads: int = 0) -> None:
        check(lib.rb_scene_build_bvh_ex(self._h, int(max_leaf), int(threads)), "build_bvh")

    def export_bvh(self) -> BVHExport:
        n = int(lib.rb_scene_num_bvh_nodes(self._h))
        bounds = np.zeros((n, 6), np.float64)
        a = np.zeros(n, np.int32)
        b = np.zeros(n, np.int32)
        leaf = np.zeros(n, np.uint8)
        ax = np.zeros(n, np.uint8)
        if n:
            check(lib.rb_scene_export_bvh(self._h, bounds.ctypes.data_as(c_double_p), a.ctypes.data_as(c_int32_p),
                                          b.ctypes.data_as(c_int32_p), leaf.ctypes.data_as(c_uint8_p),
                                          ax.ctypes.data_as(c_uint8_p)), "export_bvh")
        return BVHExport(bounds, a, b, leaf, ax, int(lib.rb_scene_bvh_root(self._h)))

    def check_wide(self) -> dict:
        """Host-only consistency check of the 4-wide copy of the built BVH
        (rb_scene_check_wide): raises on an inconsistency, returns the counts."""
        out = np.zeros(4, np.int64)
        st = lib.rb_scene_check_wide(self._h, out.ctypes.data_as(C.POINTER(C.c_int64)))
        if st != 0:
            raise RuntimeError(f"rb_scene_check_wide: {(lib.rb_last_error() or b'').decode()}")
        return {"wide_nodes": int(out[0]), "leaves_reached": int(out[1]), "binary_leaves": int(out[2]),
                "depth": int(out[3])}

    def export_order(self) -> np.ndarray:
        o = np.zeros(self.num_geometries, np.int64)
        if o.size:
            check(lib.rb_scene_export_order(self._h, o.ctypes.data_as(c_int64_p)), "export_order")
        return o

    def export_geometry(self) -> np.ndarray:
        """(n, 32) float64 rows: type, material, visible, has_normals, p[18], bmin, bmax, original index."""
        g = np.zeros((self.num_geometries, 32), np.float64)
        if g.size:
            check(lib.rb_scene_export_geometry_full(self._h, g.ctypes.data_as(c_double_p)), "export_geometry")
        return g

    def export_materials(self) -> list[MaterialDesc]:
        n = self.num_materials
        arr = (MaterialDesc * max(1, n))()
        if n:
            check(lib.rb_scene_export_materials(self._h, arr), "export_materials")
        return list(arr[:n])

    # --- device --------------------------------------------------------------------
    def upload(self, quantized: bool = False, use_bvh: bool = True, stream=None, layout: str = "as_built",
               max_leaf: int = 0, tune_depth: int = 0, probe=None, traversal_budget: int = 0,
               wide: bool = True) -> "DeviceScene":
        """layout: "as_built" (the built BVH; bit-exact primary hits), "autotune"
        (fastest of linear / groups of 8, 16 / leaf 1, 2, 4, 8 on a probe render),
        "linear", "leaf" (rebuilt with max_leaf), "groups" (the built BVH's subtrees of
        at most max_leaf primitives tested in order, no traversal stack).
        wide: the render kernels traverse a 4-wide copy of the tree (default); False
        keeps the binary tree only."""
        o = UploadOpts()
        o.quantized_bvh = int(quantized)
        o.wide_bvh = 1 if wide else -1
        o.use_bvh = int(use_bvh)
        o.layout = {"as_built": 0, "autotune": 1, "linear": 2, "leaf": 3, "groups": 4}[layout]
        o.max_leaf = int(max_leaf)
        o.tune_depth = int(tune_depth)
        o.traversal_budget = int(traversal_budget)
        keep = None
        if probe is not None:  # (frame[21], width, height): autotune on this camera
            keep = np.ascontiguousarray(probe[0], np.float64)
            o.probe_frame = keep.ctypes.data_as(c_double_p)
            o.probe_width, o.probe_height = int(probe[1]), int(probe[2])
        h = lib.rb_scene_upload(self._h, C.byref(o), stream)
        if not h:
            raise RuntimeError(f"rb_scene_upload failed: {(lib.rb_last_error() or b'').decode()}")
        return DeviceScene(h)


class DeviceScene:
    """Device-resident scene; the handle doubles as the reference's CudaScene::Scene*."""

    def __init__(self, handle) -> None:
        self.handle = handle

    @property
    def nbytes(self) -> int:
        return int(lib.rb_scene_device_bytes(self.handle))

    @property
    def layout(self) -> dict:
        k, leaf, ms = C.c_int32(0), C.c_int32(0), C.c_float(0)
        lib.rb_scene_layout_info(self.handle, C.byref(k), C.byref(leaf), C.byref(ms))
        kind = {2: "linear", 4: "groups"}.get(k.value, "bvh")
        return {"kind": kind, "leaf": leaf.value, "probe_ms": ms.value}

    @property
    def tuning(self) -> dict:
        """The autotuner's decision for this scene (rb_tuning)."""
        from ._native import Tuning
        t = Tuning()
        check(lib.rb_scene_tuning(self.handle, C.byref(t)), "rb_scene_tuning")
        return {f: getattr(t, f) for f, _ in Tuning._fields_ if f != "reserved_"}

    def traversal_faults(self, reset: bool = False) -> int:
        """Rays whose BVH traversal ran out of its step budget (0 for a well-formed tree)."""
        n = C.c_uint64(0)
        check(lib.rb_scene_traversal_faults(self.handle, C.byref(n), int(reset)), "rb_scene_traversal_faults")
        return int(n.value)

    def free(self) -> None:
        if self.handle:
            lib.rb_scene_free_device(self.handle)
            self.handle = None

    def __del__(self) -> None:
        try:
            self.free()
        except Exception:
            pass


def camera_frame(look_from, look_at, vup, vfov: float, width: int, height: int) -> np.ndarray:
    """FP64 camera frame (camera_base.hpp:76-99): rows center, pixel00, du, dv, u, v, w -> (21,)."""
    out = np.zeros(21, np.float64)
    lib.rb_camera_frame(_d3(look_from), _d3(look_at), _d3(vup), float(vfov), int(width), int(height),
                        out.ctypes.data_as(c_double_p))
    return out
