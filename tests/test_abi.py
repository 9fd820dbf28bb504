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


def test_camera_frame_bit_exact_against_camera_base():
    """rb_camera_frame equals the reference's own CameraBase::buildFrame
    (camera_base.hpp:47-99, compiled from its sources into oracle/_ref) bit for
    bit on every workload camera, orbit views and odd aspect ratios."""
    from oracle import refbind
    if not refbind.host_available():
        pytest.skip("reference drivers (oracle/_ref) not built")
    from rayon_b200 import scenes
    cams = [(scenes.one_weekend().camera, 400, 225), (scenes.cornell().camera, 512, 512),
            (scenes.icospheres(count=1, level=0).camera, 1920, 1080)]
    cams += [(v, 1280, 720) for v in scenes.sdf_field(count=2).views]
    cams += [(scenes.orbit(scenes.cornell().camera, a), 256, 256) for a in np.linspace(0.0, 6.0, 7)]
    cams += [(scenes.Camera((1.5, -2.0, 7.25), (0.1, 0.2, -0.3), (0.2, 1.0, 0.1), 73.0), 33, 517)]
    for c, w, h in cams:
        np.testing.assert_array_equal(c.frame(w, h), refbind.camera_frame(c, w, h))


def test_fault_injection_sites_are_checked():
    assert lib.rb_inject_alloc_failures(b"no_such_site", 1) == -1
    assert lib.rb_inject_alloc_failures(b"server_job", -2) == -1
    assert lib.rb_inject_alloc_failures(b"server_job", 0) == 0
    assert lib.rb_inject_alloc_failures(b"wavefront_queue", 0) == 0
