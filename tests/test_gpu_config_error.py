"""The error of each benchmark configuration against the FP64 oracle, at the
configuration's own size and settings, and the reference CUDA renderer's error
at the same settings beside it.

Ground truth: the oracle's mean radiance on 1024 seeded pixels of the full
frame at 16-32k spp (tests/golden/oracle_px_<case>.npz, make_golden.py
--oracle). Ours: one frame of the configuration (its resolution, spp and
depth; the SDF field through the wavefront engine the benchmark uses). The
estimator is unbiased, so the RMSE over those pixels must be the sample
noise of one frame: two frames on independent sample streams differ by
sqrt(2) times it. The reference's renderPixelsCUDAAccumulative renders the
same frame (configurations it can render: the One-Weekend scene with depth of
field and the Cornell box) and must show the same error: equal RMSE at equal
spp."""
import ctypes as C
import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from cases import ORACLE_PX_CASES  # noqa: E402

from oracle import refbind  # noqa: E402
from rayon_b200 import render  # noqa: E402

GOLDEN = Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu


def _ours(spec, fr, base):
    w, h = spec.width, spec.height
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload()
    if spec.name == "sdf_field":
        img = render.render_views_wavefront(ds, [fr], w, h, spec.spp, spec.depth, background=spec.background,
                                            sample_base=base, queue_capacity=1 << 22)[0]
    else:
        img = render.render_accumulate(ds, fr, w, h, spec.spp, spec.depth, background=spec.background, dof=spec.dof,
                                       sample_base=base)
    ds.free()
    return img.reshape(-1, 3) / spec.spp


def _reference(spec, fr):
    L = refbind.cuda()
    rs = refbind.RefCudaScene(spec)
    dof = spec.dof or (0.1, 10.0)
    L.refc_set_globals(1.0, spec.background, 0.8, 1.5, int(spec.dof is not None), dof[0], dof[1])
    w, h = spec.width, spec.height
    acc = np.zeros(w * h * 3, np.float32)
    frc = np.ascontiguousarray(fr, np.float64)
    secs = L.refc_render(rs.h, w, h, frc.ctypes.data_as(C.POINTER(C.c_double)), spec.spp, 1, spec.depth,
                         acc.ctypes.data_as(C.POINTER(C.c_float)))
    L.refc_set_globals(1.0, 1.0, 0.8, 1.5, 0, 0.1, 10.0)
    rs.free()
    assert secs >= 0
    return acc.reshape(-1, 3).astype(np.float64) / spec.spp


def _rmse(a, b):
    return float(np.sqrt(((a - b) ** 2).mean()))


@pytest.mark.parametrize("name", list(ORACLE_PX_CASES))
def test_configuration_error_vs_fp64_oracle(cuda, name):
    f = GOLDEN / f"oracle_px_{name}.npz"
    g = np.load(f)
    spec = ORACLE_PX_CASES[name][0]()
    w, h = spec.width, spec.height
    assert (w, h) == (int(g["width"]), int(g["height"]))
    fr = spec.camera.frame(w, h)
    px, truth = g["pixels"], g["mean"]
    a = _ours(spec, fr, 0)[px]
    b = _ours(spec, fr, 1 << 20)[px]
    err = _rmse(a, truth)
    noise = _rmse(a, b) / np.sqrt(2.0)        # one frame's sample noise
    out = {"config": name, "spp": spec.spp, "rmse_vs_oracle": err, "frame_noise": noise,
           "oracle_spp": int(g["spp"]), "pixels": int(px.shape[0])}
    if name in ("one_weekend", "cornell") and refbind.cuda_available():
        r = _reference(spec, fr)[px]
        out["reference_rmse_vs_oracle"] = _rmse(r, truth)
    print("CONFIG_ERROR", json.dumps(out))
    dest = os.environ.get("RAYON_CONFIG_ERROR_OUT")
    if dest:
        with open(dest, "a") as fh:
            fh.write(json.dumps(out) + "\n")
    # unbiased against the oracle: the error is the frame's own noise
    assert err < 1.25 * noise + 1e-3, out
    if "reference_rmse_vs_oracle" in out:
        # equal RMSE at equal spp
        assert err < 1.25 * out["reference_rmse_vs_oracle"] + 1e-3, out
        assert out["reference_rmse_vs_oracle"] < 1.25 * err + 1e-3, out
