"""ctypes wrapper of the FP64 oracle (oracle/rb_oracle.cpp). Test infrastructure only."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .build import OUT, build_oracle

_lib = None
dp = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
u8p = C.POINTER(C.c_uint8)


class OrcGlobals(C.Structure):
    _fields_ = [("light", C.c_double), ("background", C.c_double), ("fuzz", C.c_double), ("glass_ior", C.c_double),
                ("dof", C.c_int), ("aperture", C.c_double), ("focus", C.c_double), ("nee", C.c_int)]


@dataclass
class Globals:
    """Reference __constant__ defaults (renderer_cuda_device.cu:18-26)."""
    light: float = 1.0
    background: float = 1.0
    fuzz: float = 0.8
    glass_ior: float = 1.5
    dof: bool = False
    aperture: float = 0.1
    focus: float = 10.0
    nee: bool = False

    def c(self) -> OrcGlobals:
        return OrcGlobals(self.light, self.background, self.fuzz, self.glass_ior, int(self.dof), self.aperture,
                          self.focus, int(self.nee))


def lib():
    global _lib
    if _lib is None:
        from .refbind import RefMaterial as MaterialDesc
        if not OUT.exists():
            build_oracle()
        L = C.CDLL(str(OUT))
        L.orc_scene_create.restype = C.c_void_p
        L.orc_scene_create.argtypes = [dp, C.c_int64, C.POINTER(MaterialDesc), C.c_int, dp, i32p, i32p, u8p, u8p,
                                       C.c_int64, C.c_int]
        L.orc_scene_destroy.argtypes = [C.c_void_p]
        L.orc_scene_set_sdf.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_double]
        L.orc_primary.argtypes = [C.c_void_p, C.c_int, C.c_int, dp, i32p, dp, i64p, C.c_int]
        L.orc_render.argtypes = [C.c_void_p, C.c_int, C.c_int, dp, i32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.POINTER(OrcGlobals), C.c_uint32, C.c_uint32, dp, C.c_int, i64p]
        _lib = L
    return _lib


class OracleScene:
    """FP64 scene built from a SceneDescription whose BVH has been built."""

    def __init__(self, sc, use_bvh: bool = True, sdf: tuple | None = None) -> None:
        """sdf = (blend radius k, max steps, epsilon) for scenes with SDF primitives."""
        b = sc.export_bvh()
        self._init(sc.export_geometry(), sc.export_materials(), b if use_bvh else None, sdf)

    @classmethod
    def from_arrays(cls, spec, sdf: tuple | None = None) -> "OracleScene":
        """A scene straight from workload arrays (materials, kinds, params,
        mats in insertion order), traversed by linear scan: no BVH and no
        call into this project's library."""
        o = cls.__new__(cls)
        kinds = np.asarray(spec.kinds)
        g = np.zeros((kinds.shape[0], 32), np.float64)
        # geometry kinds of the workload arrays -> Scene::GeometryType numbering
        g[:, 0] = np.choose(kinds, [0, 1, 4, 6])
        g[:, 1] = spec.mats
        g[:, 2] = 1.0
        g[:, 4:22] = spec.params
        g[:, 31] = np.arange(kinds.shape[0])
        o._init(g, list(spec.materials), None, sdf)
        return o

    def _init(self, geoms, mats, b, sdf) -> None:
        from .refbind import RefMaterial, as_ref_material
        L = lib()
        self.geoms = np.ascontiguousarray(geoms, np.float64)
        self._mats = (RefMaterial * max(1, len(mats)))(*[as_ref_material(m) for m in mats])
        self._b = b
        if b is not None:
            self.h = L.orc_scene_create(self.geoms.ctypes.data_as(dp), self.geoms.shape[0], self._mats, len(mats),
                                        b.bounds.ctypes.data_as(dp), b.a.ctypes.data_as(i32p),
                                        b.b.ctypes.data_as(i32p), b.is_leaf.ctypes.data_as(u8p),
                                        b.split_axis.ctypes.data_as(u8p), b.a.shape[0], b.root)
        else:
            self.h = L.orc_scene_create(self.geoms.ctypes.data_as(dp), self.geoms.shape[0], self._mats, len(mats),
                                        None, None, None, None, None, 0, -1)
        if sdf is not None:
            L.orc_scene_set_sdf(self.h, float(sdf[0]), int(sdf[1]), float(sdf[2]))

    def primary(self, frame: np.ndarray, w: int, h: int, threads: int = 0):
        ids = np.zeros(w * h, np.int32)
        t = np.zeros(w * h, np.float64)
        cnt = np.zeros(2, np.int64)
        fr = np.ascontiguousarray(frame, np.float64)
        lib().orc_primary(self.h, w, h, fr.ctypes.data_as(dp), ids.ctypes.data_as(i32p), t.ctypes.data_as(dp),
                          cnt.ctypes.data_as(i64p), threads)
        return ids.reshape(h, w), t.reshape(h, w), cnt

    def render(self, frame, w: int, h: int, spp: int, depth: int, globals_: Globals, seed: int, salt: int = 0,
               sample_base: int = 0, pixels=None, threads: int = 0):
        """Per-pixel radiance sums (npix, 3) FP64 and 14 work counters: nodes visited,
        primitives tested, segments, paths, shadow rays; primitive tests by kind
        (sphere, rectangle, triangle, SDF); shading events by class (Lambert,
        mirror / rough mirror, glass, emitter / constant / normals, GGX
        conductor / thin film / clear coat)."""
        fr = np.ascontiguousarray(frame, np.float64)
        px = None if pixels is None else np.ascontiguousarray(pixels, np.int32)
        n = w * h if px is None else px.shape[0]
        out = np.zeros((n, 3), np.float64)
        cnt = np.zeros(14, np.int64)
        g = globals_.c()
        lib().orc_render(self.h, w, h, fr.ctypes.data_as(dp), None if px is None else px.ctypes.data_as(i32p), n,
                         spp, sample_base, depth, C.byref(g), seed, salt, out.ctypes.data_as(dp), threads,
                         cnt.ctypes.data_as(i64p))
        return out, cnt

    def __del__(self) -> None:
        if getattr(self, "h", None):
            lib().orc_scene_destroy(self.h)
            self.h = None
