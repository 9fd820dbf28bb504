"""B200-native (sm_100a) path-tracing render path, a drop-in for RayON's CUDA renderer.

The product is the native library rayon_b200/_lib/librayon_b200.so (C-ABI in
include/rayon_b200.h). This package is the thin Python plumbing used by the
tests and the benchmark; importing it fails loudly if the library is missing.
"""
from . import _native  # noqa: F401  (loads the library or raises)
from ._native import lib, last_error  # noqa: F401
from .scene import SceneDescription, DeviceScene, camera_frame  # noqa: F401

__all__ = ["lib", "last_error", "SceneDescription", "DeviceScene", "camera_frame"]
