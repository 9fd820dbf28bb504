"""The C-ABI library loads and exports every entry point declared in include/*.h;
argument errors come back as status codes with a message (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

import rayon_b200
from rayon_b200 import scene as S
from rayon_b200._native import lib

INCLUDE = Path(__file__).resolve().parent.parent / "include"


def declared_functions():
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            pre = text[max(0, m.start() - 80):m.start()]
            if name in ("sizeof", "RB_DEFAULT", "if", "while", "for", "return") or "#define" in pre.splitlines()[-1:][0:1]:
                continue
            names.add(name)
    return names


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    # the reference's drop-in group must be there
    for n in ["renderPixelsCUDAAccumulative", "initCudaStreams", "cleanupCudaStreams", "freeDeviceRandomStates",
              "freeDeviceAccumBuffer", "resetDeviceAccumBuffer", "setLightIntensity", "setBackgroundIntensity",
              "setMetalFuzziness", "setGlassRefractionIndex", "setDOFEnabled", "setDOFAperture",
              "setDOFFocusDistance", "convertAccumToDisplayCUDA", "allocateAdaptiveBuffer", "resetAdaptiveBuffer",
              "freeAdaptiveBuffer", "countConvergedPixels", "renderSampleHeatmapCUDA"]:
        assert n in names, n
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_errors_are_status_codes():
    assert lib.rb_scene_build_bvh_ex(None, 4, 0) < 0
    sc = S.SceneDescription()
    assert lib.rb_scene_build_bvh_ex(sc.handle, 0, 0) < 0
    assert "max_leaf" in rayon_b200.last_error()
    assert lib.rb_scene_set_visible(sc.handle, 5, 1) < 0
    assert lib.rb_primary_hits(None, 4, 4, None, None, None, None) < 0


def test_camera_frame_matches_reference_formula():
    # CameraBase::initialize (camera_base.hpp:76-99) evaluated independently
    lf, la, vup, vfov, w, h = np.array([13., 2, 3]), np.zeros(3), np.array([0., 1, 0]), 20.0, 400, 225
    fr = S.camera_frame(lf, la, vup, vfov, w, h).reshape(7, 3)
    focal = np.linalg.norm(lf - la)
    hh = np.tan(np.deg2rad(vfov) / 2)
    vh = 2 * hh * focal
    vw = vh * w / h
    ww = (lf - la) / focal
    u = np.cross(vup, ww)
    u /= np.linalg.norm(u)
    v = np.cross(ww, u)
    du, dv = vw * u / w, -vh * v / h
    p00 = lf - focal * ww - vw * u / 2 + vh * v / 2 + 0.5 * (du + dv)
    np.testing.assert_allclose(fr[1], p00, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(fr[2], du, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(fr[3], dv, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(fr[4:7], np.stack([u, v, ww]), atol=1e-15)
