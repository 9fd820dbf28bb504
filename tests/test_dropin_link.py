"""The drop-in boundary at link level (CPU): RayON's unmodified offline CUDA
renderer (gpu_renderers/renderer_cuda_host.hpp, driven through
render/render_coordinator.cpp) and the adapter
rayon_b200/adapter/rayon_b200_adapter.cpp, compiled against the reference's
own headers and linked with --no-undefined to librayon_b200.so and to no
object of the reference's .cu sources (oracle/ref/Makefile, target
librayon_dropin.so). Every symbol the renderer and the adapter import must be
defined by this library, and the result must load."""
import ctypes as C
import os
import subprocess
from pathlib import Path

import pytest

from oracle import build as obuild

ROOT = Path(__file__).resolve().parent.parent
DROPIN = ROOT / "oracle" / "_ref" / "librayon_dropin.so"
LIB = ROOT / "rayon_b200" / "_lib" / "librayon_b200.so"


def _symbols(path, flag):
    out = subprocess.run(["nm", "-D", flag, str(path)], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


@pytest.fixture(scope="module")
def dropin():
    if (obuild.REFERENCE / "src" / "rayon").is_dir():
        r = subprocess.run(["make", "-C", str(ROOT / "oracle" / "ref"), f"REF={obuild.REFERENCE}",
                            str(DROPIN)], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    if not DROPIN.exists():
        pytest.skip("reference tree absent and oracle/_ref/librayon_dropin.so not built")
    return DROPIN


def test_renderer_links_against_this_library_only(dropin):
    imported = _symbols(dropin, "--undefined-only")
    exported = _symbols(LIB, "--defined-only")
    ours = {s for s in imported if s.startswith(("rb_", "render", "free", "set", "convert", "allocate", "count",
                                                  "reset", "init", "cleanup"))}
    # what RayON's RendererCUDA::render calls (renderer_cuda_host.hpp:35-67), plus the setter the caller uses
    for s in ("renderPixelsCUDAAccumulative", "freeDeviceRandomStates", "freeDeviceAccumBuffer",
              "setBackgroundIntensity", "rb_scene_upload", "rb_scene_free_device"):
        assert s in ours, s
    assert ours <= exported, sorted(ours - exported)
    # no reference GPU code inside: its kernels and scene builder are absent
    defined = _symbols(dropin, "--defined-only")
    assert not any(k in " ".join(defined) for k in ("renderAccKernel", "gammaCorrectKernel", "convertGeometry"))
    # the adapter defines the reference's scene-upload entry points
    assert {"_ZN5Scene16CudaSceneBuilder13buildGPUSceneERKNS_16SceneDescriptionE",
            "_ZN5Scene16CudaSceneBuilder12freeGPUSceneEPN9CudaScene5SceneE"} <= defined


def test_renderer_library_loads_with_all_symbols_bound(dropin):
    C.CDLL(str(LIB), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    L = C.CDLL(str(dropin), mode=os.RTLD_NOW)
    assert L.dropin_render_offline and L.dropin_accum_to_image
