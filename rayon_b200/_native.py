"""ctypes bindings to librayon_b200.so (the C-ABI declared in include/rayon_b200.h).

The library is loaded eagerly and the import fails loudly when it is absent:
there is no Python or CPU fallback for any render entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# RAYON_B200_LIB selects another build of the same library (e.g. one compiled
# with different -D options); the default is the in-tree build.
_LIB_PATH = Path(os.environ.get("RAYON_B200_LIB") or
                 Path(__file__).resolve().parent / "_lib" / "librayon_b200.so")


class NativeLibraryMissing(RuntimeError):
    pass


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise NativeLibraryMissing(
            f"{_LIB_PATH} is missing: run `python -c 'import __graft_entry__ as g; g.build()'` "
            "(or python rayon_b200/build.py) to compile the CUDA library")
    return C.CDLL(str(_LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)


lib = _load()

c_double_p = C.POINTER(C.c_double)
c_float_p = C.POINTER(C.c_float)
c_int32_p = C.POINTER(C.c_int32)
c_int64_p = C.POINTER(C.c_int64)
c_uint8_p = C.POINTER(C.c_uint8)
c_uint64_p = C.POINTER(C.c_uint64)
vp = C.c_void_p


class MaterialDesc(C.Structure):
    """rb_material_desc (mirrors Scene::MaterialDesc, scene_description.hpp:58-101)."""
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


class UploadOpts(C.Structure):
    _fields_ = [("quantized_bvh", C.c_int), ("use_bvh", C.c_int), ("layout", C.c_int), ("max_leaf", C.c_int),
                ("tune_depth", C.c_int), ("probe_width", C.c_int), ("probe_height", C.c_int),
                ("probe_frame", C.POINTER(C.c_double)), ("traversal_budget", C.c_int), ("wide_bvh", C.c_int)]


LAYOUT_AS_BUILT, LAYOUT_AUTOTUNE, LAYOUT_LINEAR, LAYOUT_LEAF = 0, 1, 2, 3


class RenderOpts(C.Structure):
    _fields_ = [("nee", C.c_int), ("kahan", C.c_int), ("seed", C.c_uint32), ("block_x", C.c_int),
                ("block_y", C.c_int), ("reserved", C.c_int * 4)]


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


# --- errors / version ---------------------------------------------------------
_sig("rb_last_error", C.c_char_p)
_sig("rb_version", C.c_char_p)
_sig("rb_launch_count", C.c_ulonglong)
_sig("rb_kernel_timer_enable", None, C.c_int)
_sig("rb_kernel_timer_read", C.c_int, c_double_p, c_int64_p)
_sig("rb_inject_alloc_failures", C.c_int, C.c_char_p, C.c_int)

# --- drop-in group (renderer_cuda_device.cuh:8-67) ---------------------------
_sig("initCudaStreams", None)
_sig("cleanupCudaStreams", None)
_sig("renderPixelsCUDAAccumulative", C.c_ulonglong,
     c_uint8_p, c_float_p, vp, C.c_int, C.c_int,
     C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
     C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
     C.c_int, C.c_int, C.c_int, C.POINTER(vp), C.POINTER(vp),
     C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
     vp, C.c_int, C.c_float)
_sig("freeDeviceRandomStates", None, vp)
_sig("freeDeviceAccumBuffer", None, vp)
_sig("resetDeviceAccumBuffer", None, vp, C.c_int)
for _n in ("setLightIntensity", "setBackgroundIntensity", "setMetalFuzziness", "setGlassRefractionIndex",
           "setDOFAperture", "setDOFFocusDistance"):
    _sig(_n, None, C.c_float)
_sig("setDOFEnabled", None, C.c_bool)
_sig("convertAccumToDisplayCUDA", None, vp, c_uint8_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, vp)
_sig("allocateAdaptiveBuffer", None, C.POINTER(vp), C.c_int)
_sig("resetAdaptiveBuffer", None, vp, C.c_int)
_sig("freeAdaptiveBuffer", None, vp)
_sig("countConvergedPixels", C.c_int, vp, C.c_int)
_sig("renderSampleHeatmapCUDA", None, vp, c_uint8_p, C.c_int, C.c_int, C.c_int, C.c_int)

# --- scene -----------------------------------------------------------------
_sig("rb_material_default", None, C.POINTER(MaterialDesc))
_sig("rb_scene_create", vp)
_sig("rb_scene_destroy", None, vp)
_sig("rb_scene_add_material", C.c_int, vp, C.POINTER(MaterialDesc))
_sig("rb_scene_add_sphere", C.c_int, vp, c_double_p, C.c_double, C.c_int)
_sig("rb_scene_add_displaced_sphere", C.c_int, vp, c_double_p, C.c_double, C.c_int, C.c_float, C.c_int)
_sig("rb_scene_add_rectangle", C.c_int, vp, c_double_p, c_double_p, c_double_p, C.c_int)
_sig("rb_scene_add_triangle", C.c_int, vp, c_double_p, c_double_p, c_double_p, C.c_int)
_sig("rb_scene_add_triangle_with_normals", C.c_int, vp, c_double_p, c_double_p, c_double_p,
     c_double_p, c_double_p, c_double_p, C.c_int)
_sig("rb_scene_add_sdf", C.c_int, vp, C.c_int, c_double_p, c_double_p, c_double_p, C.c_int)
_sig("rb_scene_add_spheres", C.c_int64, vp, c_double_p, c_int32_p, C.c_int, C.c_int64)
_sig("rb_scene_add_triangles", C.c_int64, vp, c_double_p, c_double_p, c_int32_p, C.c_int, C.c_int64)
_sig("rb_scene_load_obj", C.c_int64, vp, C.c_char_p, C.c_int, c_double_p, c_double_p)
_sig("rb_scene_set_visible", C.c_int, vp, C.c_int64, C.c_int)
_sig("rb_scene_num_geometries", C.c_int64, vp)
_sig("rb_scene_num_materials", C.c_int, vp)
_sig("rb_scene_set_sdf_blend", C.c_int, vp, C.c_float, C.c_int, C.c_float)
_sig("rb_scene_build_bvh", C.c_int, vp)
_sig("rb_scene_build_bvh_ex", C.c_int, vp, C.c_int, C.c_int)
_sig("rb_scene_num_bvh_nodes", C.c_int64, vp)
_sig("rb_scene_bvh_root", C.c_int, vp)
_sig("rb_scene_export_bvh", C.c_int, vp, c_double_p, c_int32_p, c_int32_p, c_uint8_p, c_uint8_p)
_sig("rb_scene_export_order", C.c_int, vp, c_int64_p)
_sig("rb_scene_export_geometry_full", C.c_int, vp, c_double_p)
_sig("rb_scene_export_materials", C.c_int, vp, C.POINTER(MaterialDesc))
_sig("rb_camera_frame", None, c_double_p, c_double_p, c_double_p, C.c_double, C.c_int, C.c_int, c_double_p)

# --- device scene / rendering ----------------------------------------------------
_sig("rb_scene_upload", vp, vp, C.POINTER(UploadOpts), vp)
_sig("rb_scene_free_device", None, vp)
_sig("rb_scene_device_bytes", C.c_int64, vp)
_sig("rb_scene_traversal_faults", C.c_int, vp, c_uint64_p, C.c_int)
_sig("rb_scene_check_wide", C.c_int, vp, C.POINTER(C.c_int64))
_sig("rb_scene_layout_info", C.c_int, vp, c_int32_p, c_int32_p, c_float_p)


class Tuning(C.Structure):
    """rb_tuning: what the autotuner chose for a scene."""
    _fields_ = [("layout", C.c_int), ("leaf", C.c_int), ("blocks_per_sm", C.c_int), ("block_x", C.c_int),
                ("block_y", C.c_int), ("short_stack", C.c_int), ("wavefront_queue", C.c_int),
                ("probe_ms", C.c_float), ("from_cache", C.c_int), ("reserved_", C.c_int * 3)]


_sig("rb_scene_tuning", C.c_int, vp, C.POINTER(Tuning))
_sig("rb_primary_hits", C.c_int, vp, C.c_int, C.c_int, c_double_p, vp, vp, vp)
_sig("rb_get_render_opts", None, C.POINTER(RenderOpts))
_sig("rb_set_render_opts", None, C.POINTER(RenderOpts))
_sig("rb_render_accumulate", C.c_int, vp, C.c_int, C.c_int, c_double_p, C.c_int, C.c_int, C.c_int,
     vp, vp, vp, vp)
_sig("rb_render_wavefront", C.c_int, vp, C.c_int, C.c_int, c_double_p, C.c_int, C.c_int, C.c_int, vp, C.c_int,
     vp, vp)
_sig("rb_render_views", C.c_int, vp, C.c_int, C.c_int, C.c_int, c_double_p, C.c_int, C.c_int, C.c_int, vp, vp, vp)
_sig("rb_render_views_wavefront", C.c_int, vp, C.c_int, C.c_int, C.c_int, c_double_p, C.c_int, C.c_int, C.c_int, vp,
     C.c_int, vp, vp)


def last_error() -> str:
    return (lib.rb_last_error() or b"").decode()


def check(status: int, what: str = "") -> int:
    if status < 0:
        raise RuntimeError(f"{what} failed ({status}): {last_error()}")
    return status


# --- batched engine / serving loop ---------------------------------------------
class JobRequest(C.Structure):
    _fields_ = [("scene", C.c_int), ("width", C.c_int), ("height", C.c_int), ("spp", C.c_int),
                ("max_depth", C.c_int), ("frame", C.c_double * 21), ("light_intensity", C.c_float),
                ("background_intensity", C.c_float), ("metal_fuzziness", C.c_float), ("glass_ior", C.c_float),
                ("dof_enabled", C.c_int), ("dof_aperture", C.c_float), ("dof_focus", C.c_float), ("nee", C.c_int),
                ("seed", C.c_uint32), ("fp64_accum", C.c_int), ("arrival_time", C.c_double),
                ("converge_threshold", C.c_float), ("converge_min_spp", C.c_int), ("converge_fraction", C.c_float),
                ("converge_pad", C.c_int)]


class ServerOpts(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_int64), ("max_active_jobs", C.c_int), ("paths_per_iteration", C.c_int64),
                ("max_spp_per_iteration", C.c_int), ("use_graph", C.c_int), ("frames_every", C.c_int),
                ("occupancy", C.c_int), ("wavefront_field", C.c_int), ("target_iteration_ms", C.c_float),
                ("per_frame_classes", C.c_int)]


class JobStatus(C.Structure):
    _fields_ = [("state", C.c_int), ("spp_done", C.c_int), ("t_arrival", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("device_bytes", C.c_int64), ("error", C.c_int), ("reserved_", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("jobs_done", C.c_int64), ("jobs_rejected", C.c_int64), ("iterations", C.c_int64),
                ("frames", C.c_int64), ("paths", C.c_int64), ("segments", C.c_int64),
                ("device_seconds", C.c_double), ("wall_seconds", C.c_double), ("peak_device_bytes", C.c_int64),
                ("p50_latency", C.c_double), ("p99_latency", C.c_double), ("mean_latency", C.c_double),
                ("quantum_paths", C.c_int64), ("last_iteration_ms", C.c_double)]


_sig("rb_job_default", None, C.POINTER(JobRequest))
_sig("rb_server_default_opts", None, C.POINTER(ServerOpts))
_sig("rb_server_create", vp, C.POINTER(ServerOpts), vp)
_sig("rb_server_destroy", None, vp)
_sig("rb_server_add_scene", C.c_int, vp, vp)
_sig("rb_server_submit", C.c_int64, vp, C.POINTER(JobRequest))
_sig("rb_server_step", C.c_int, vp)
_sig("rb_server_job_status", C.c_int, vp, C.c_int64, C.POINTER(JobStatus))
_sig("rb_server_fetch", C.c_int, vp, C.c_int64, c_float_p, c_uint8_p)
_sig("rb_server_release", C.c_int, vp, C.c_int64)
_sig("rb_server_run_trace", C.c_int, vp, C.POINTER(JobRequest), C.c_int64, C.c_int, C.c_int, c_double_p)
_sig("rb_server_get_stats", C.c_int, vp, C.POINTER(ServerStats))
_sig("convertAccumToDisplayNoAlloc", C.c_int, vp, c_uint8_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, vp)
