"""Benchmark of the B200 render path (one JSON line on rank 0).

Default workload (the one the metric is quoted on): the Cornell box (512x512,
256 spp, max depth 16, FP32 radiance with Kahan-compensated accumulation,
background 0). One step = one full frame: 512*512*256 = 67.1 M primary paths.
`value` = Mpaths/s with the scene and the accumulation buffers resident in HBM
(device time, CUDA events per step on the launching stream, L2 flushed between
steps). `e2e` = the same frames through the drop-in C-ABI call exactly as
RayON's offline renderer makes it (renderer_cuda_host.hpp:23-74): scene upload
from host memory, five renderPixelsCUDAAccumulative calls with a host float3
accumulation buffer (uploaded on the first call, downloaded after every call),
free.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload cornell|one_weekend|icospheres|sdf_field]

The other workloads: one_weekend (400x225, 32 spp, depth 10, depth of field),
icospheres (5.24 M triangles, 1920x1080, 64 spp, depth 8) and sdf_field (256
SDF primitives in a smooth union, 1280x720, 128 spp, depth 8, 16 orbit views
per step in ONE launch of rb_render_views); their e2e is scene upload + render
+ accumulation readback through the public API.

--impl reference times the reference's own CPU renderer (RendererCPUParallel,
compiled from the reference sources into oracle/_ref/) on the host cores on a
bounded sample of the same frame (the FP64 oracle port where that renderer
cannot render the scene), and the reference's own CUDA renderer built for
sm_100a on the same frame.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mpaths/s (Cornell box 512x512, 256 spp, depth 16)"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms. Started
    before the warm-up so that sampling is running when the timed region
    begins; mark() brackets the timed region and summary() keeps the samples
    taken inside it (or within 0.5 s of it when the region is shorter than
    the sampling period)."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def mark(self, start: bool) -> None:
        if start:
            self.t0 = time.time()
        else:
            self.t1 = time.time()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, keep: bool = False):
        import datetime
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 10:
                try:
                    p[0] = datetime.datetime.strptime(p[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    continue
                rows.append(p)
        if not keep:
            os.unlink(self.path)
        window = "timed region"
        if self.t0 is not None and self.t1 is not None:
            inside = [r for r in rows if self.t0 <= r[0] <= self.t1]
            if not inside:
                inside = [r for r in rows if self.t0 - 0.5 <= r[0] <= self.t1 + 0.5]
                window = "timed region +- 0.5 s"
            rows = inside
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        num = lambda v: v.replace(".", "").isdigit()  # noqa: E731
        sm = [float(r[2]) for r in rows if num(r[2])]
        mx = [float(r[3]) for r in rows if num(r[3])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "window": window}


def measured_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return json.loads(f.read_text()), "measured"
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


# Committed ncu summary of each workload's dominant kernel (profiles/): the
# capture of the same launch the bench times (same frame, same spp).
PROFILE = {"cornell": "k_render_cornell.txt", "one_weekend": "k_render_one_weekend.txt",
           "icospheres": "k_render_icospheres.txt", "sdf_field": "k_wf_march_sdf_field.txt"}
SMS, SCHEDULERS = 148, 4
# Algorithmic work per traced segment (the unit of the roofline's achieved
# figure): FLOPs per box test, per primitive test by kind and per shading
# event by material class, and the scene bytes a test reads in this project's
# layout (a 64 B node holds two boxes: 32 B per box test; 48 B primitive
# records, of which sphere 16 B, rectangle and triangle 36 B are geometry).
FLOPS_BOX, FLOPS_PRIM, FLOPS_SHADE = 24, (20, 30, 27, 30), (40, 45, 60, 5, 150)
BYTES_BOX, BYTES_PRIM = 32, (16, 36, 36, 80)


def d4_work(workload: str):
    """Per-segment algorithmic FLOPs and scene bytes from the FP64 oracle's
    work counters on 1024 pixels of the workload's frame at high spp (the
    reference-ordered BVH, so independent of this implementation's traversal
    order), read from the committed fixture tests/golden/oracle_px_<workload>.npz
    (made by tests/golden/make_golden.py --oracle)."""
    f = ROOT / "tests" / "golden" / f"oracle_px_{workload}.npz"
    if not f.exists():
        return None
    c = np.load(f)["counters"].astype(np.float64)
    if c.shape[0] < 14 or c[2] <= 0:
        return None
    seg = c[2]
    box, kinds, shades = c[0] / seg, c[5:9] / seg, c[9:14] / seg
    flops = FLOPS_BOX * box + float(np.dot(FLOPS_PRIM[:3], kinds[:3])) + float(np.dot(FLOPS_SHADE, shades))
    scene_bytes = BYTES_BOX * box + float(np.dot(BYTES_PRIM, kinds))
    return {"flops_per_segment": flops, "scene_bytes_per_segment": scene_bytes,
            "box_tests_per_segment": box, "prim_tests_per_segment": dict(zip(("sphere", "rect", "tri", "sdf"),
                                                                              kinds.tolist())),
            "shades_per_segment": dict(zip(("lambert", "mirror", "glass", "emitter", "ggx_film_coat"),
                                           shades.tolist())),
            "segments_per_path_oracle": seg / c[3],
            "note": ("oracle counters of the reference-ordered BVH on 1024 pixels of this frame; the SDF field's "
                     "march evaluations are not counted" if workload == "sdf_field" else
                     "oracle counters of the reference-ordered BVH on 1024 pixels of this frame")}


def roofline(workload, peaks, peaks_kind, sm_mhz, t_ms, kernel_ms, segs, npaths, npx, small=False):
    """The dominant kernel against the roof that binds it. The render kernels
    are bound by instruction issue (the scene of Cornell, One-Weekend and the
    SDF field stays in L1/L2; DRAM carries only the accumulation state), so
    achieved = warp instructions per launch (ncu sm__inst_executed.sum of the
    same launch, committed under profiles/) / the kernel's live duration (CUDA
    events on its stream, rb_kernel_timer_*), peak = 148 SMs x 4 schedulers x
    one warp instruction per clock at the SM clock sampled during the timed
    steps. The HBM figures (accumulation state; ncu DRAM traffic) and the
    algorithmic FLOP rate (d4_work) stand beside it."""
    prof = {} if small else profiled_figures(PROFILE.get(workload, ""))
    k_ms = kernel_ms if kernel_ms else t_ms * float(prof.get("kernel_share_of_step", 1.0))
    ks = k_ms * 1e-3
    acc_bytes = 64 * npx                          # FP32 sums + Kahan terms, read and written once per launch
    hbm = {"achieved": acc_bytes / ks / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s",
           "frac": acc_bytes / ks / 1e9 / peaks["hbm_gbs"], "algorithmic_bytes_per_launch": acc_bytes,
           "traffic_ncu": prof.get("dram_bytes_per_launch"), "peak_kind": f"{peaks_kind} HBM copy bandwidth"}
    out = {"kernel": prof.get("kernel", "k_render"), "kernel_ms": k_ms,
           "kernel_ms_source": "live CUDA events around each launch" if kernel_ms else
           "step time x the kernel's share of the step (ncu launch list)",
           "traffic": prof.get("dram_bytes_per_launch"), "hbm": hbm}
    inst = prof.get("inst_executed_per_launch")
    per_step = prof.get("inst_executed_per_step")
    if not per_step and prof.get("inst_executed_per_path"):
        # warp instructions per path from a smaller capture of the same
        # workload, times this step's paths (the count grows with the paths)
        per_step = prof["inst_executed_per_path"] * npaths
    if not inst and per_step:
        # an engine of many launches (the wavefront engine): every warp
        # instruction of its kernels in one timed step over the step's device time
        ks = t_ms * 1e-3
        out["kernel_ms"] = t_ms
        out["kernel_ms_source"] = "the timed step (all of the engine's launches)"
        peak = SMS * SCHEDULERS * sm_mhz * 1e6 / 1e9
        ach = per_step / ks / 1e9
        out.update({"bound": "issue", "achieved": ach, "peak": peak, "unit": "Gwarp-inst/s", "frac": ach / peak,
                    "peak_kind": f"148 SMs x 4 schedulers x 1 warp-instruction/clock at the sampled {sm_mhz:.0f} MHz",
                    "inst_executed_per_step": per_step, "ncu_case": prof.get("ncu_case"),
                    "inst_executed_per_path": prof.get("inst_executed_per_path"),
                    "kernel": prof.get("kernel", "wavefront engine")})
    elif inst:
        peak = SMS * SCHEDULERS * sm_mhz * 1e6 / 1e9
        ach = inst / ks / 1e9
        out.update({"bound": "issue", "achieved": ach, "peak": peak, "unit": "Gwarp-inst/s", "frac": ach / peak,
                    "peak_kind": f"148 SMs x 4 schedulers x 1 warp-instruction/clock at the sampled {sm_mhz:.0f} MHz",
                    "inst_executed_per_launch": inst,
                    "lane_efficiency_ncu": prof.get("lane_efficiency_ncu"),
                    "issue_active_frac_ncu": prof.get("issue_active_frac_ncu"),
                    "ncu_case": prof.get("ncu_case")})
    else:
        out.update({"bound": "hbm", "achieved": hbm["achieved"], "peak": hbm["peak"], "unit": "GB/s",
                    "frac": hbm["frac"], "peak_kind": hbm["peak_kind"],
                    "note": "no ncu instruction count of this launch committed; HBM is not the binding roof"})
    for k in ("l2_gbs_ncu", "dram_gbs_ncu"):
        if k in prof:
            out[k] = prof[k]
    w = d4_work(workload)
    if w:
        fp32_peak = SMS * 128 * 2 * sm_mhz * 1e6 / 1e12
        tflops = w["flops_per_segment"] * segs / ks / 1e12
        w.update({"tflops": tflops, "fp32_peak_tflops_at_clock": fp32_peak, "frac_fp32_peak": tflops / fp32_peak,
                  "scene_gbs_touched": w["scene_bytes_per_segment"] * segs / ks / 1e9})
        if prof.get("dram_bytes_per_launch"):
            w["dram_traffic_over_scene_bytes"] = prof["dram_bytes_per_launch"] / (w["scene_bytes_per_segment"] * segs)
        out["algorithmic"] = w
    return out


def config_error(workload, step, acc, engine, nviews, npx, spp, w, h):
    """RMSE of one frame at the workload's own settings against the FP64
    oracle's mean on the 1024 seeded pixels of tests/golden/oracle_px_<workload>.npz
    (view 0 for the multi-view workload), and the frame's sample noise on
    those pixels is what an unbiased renderer shows."""
    import torch
    f = ROOT / "tests" / "golden" / f"oracle_px_{workload}.npz"
    if not f.exists():
        return None
    g = np.load(f)
    px, truth = g["pixels"], g["mean"]
    if int(g["width"]) != w or int(g["height"]) != h:
        return None
    acc.zero_()
    step(1 << 20)
    torch.cuda.synchronize()
    if engine == "wavefront":
        img = acc[0, :, :3].cpu().numpy().astype(np.float64)
    else:
        a = acc[0].cpu().numpy().astype(np.float64)
        img = a[0, :, :3] - a[1, :, :3]
    est = img[px] / spp
    return {"rmse": float(np.sqrt(((est - truth) ** 2).mean())), "pixels": int(px.shape[0]),
            "oracle_spp": int(g["spp"]), "frame_spp": spp,
            "note": "one frame at the configuration's spp vs the FP64 oracle's high-spp mean on a seeded pixel "
                    "subset (view 0 where the step renders several)"}


def profiled_figures(name: str) -> dict:
    """The `key: value` lines (unindented) of a committed ncu summary under
    profiles/, numbers as floats."""
    out = {}
    f = ROOT / "profiles" / name
    if not f.exists():
        return out
    for line in f.read_text().splitlines():
        if not line or line[0].isspace() or ":" not in line:
            continue
        k, v = (s.strip() for s in line.split(":", 1))
        if not v:
            continue
        try:
            out[k] = float(v)
        except ValueError:
            out[k] = v
    return out


def _ref_spec(workload: str):
    """The workload as plain arrays (oracle/workloads.py, identical to
    rayon_b200/scenes.py by test), for code that drives only the reference."""
    from oracle import workloads
    return workloads.WORKLOADS[workload]()


def _port_sample(spec, cam, budget_s: float):
    """The FP64 oracle (this project's CPU restatement of the path, all host
    threads, linear scan over the workload arrays) on a seeded subset of the
    frame's pixels at full spp, scaled to about budget_s seconds. Returns
    (Mpaths/s, threads, description)."""
    from oracle.oracle import Globals, OracleScene
    w, h = spec.width, spec.height
    o = OracleScene.from_arrays(spec, sdf=(spec.sdf_blend, spec.sdf_steps, spec.sdf_eps))
    fr = cam.frame(w, h)
    g = Globals(background=spec.background, dof=spec.dof is not None,
                aperture=spec.dof[0] if spec.dof else 0.1, focus=spec.dof[1] if spec.dof else 10.0)
    rng = np.random.default_rng(5)
    n = 16
    t = 0.0
    while True:
        px = rng.choice(w * h, size=n, replace=False).astype(np.int32)
        t0 = time.perf_counter()
        o.render(fr, w, h, spec.spp, spec.depth, g, seed=1, pixels=px)
        t = time.perf_counter() - t0
        if t > budget_s / 4 or n >= w * h:
            break
        n = min(w * h, int(n * max(2.0, budget_s / 4 / max(t, 1e-3))))
    threads = os.cpu_count() or 1
    return n * spec.spp / t / 1e6, threads, (f"FP64 oracle port (linear scan), {n} seeded pixels of the {w}x{h} "
                                             f"frame at {spec.spp} spp ({n * spec.spp} paths, {t:.1f} s)")


class RefCpuSample:
    """The reference's own CPU renderer (RendererCPUParallel, compiled from its
    sources into oracle/_ref, all host threads) on a bounded sample of the
    workload: the full frame at fewer spp (Cornell, One-Weekend), or the same
    camera at a reduced resolution and 1 spp (5.2 M triangles by linear scan).
    The SDF field has no reference CPU equivalent (no smooth union, no rounded
    boxes), so it is timed on the FP64 oracle port instead."""

    def __init__(self, workload: str, spec, budget_s: float):
        from oracle import refbind
        self.workload, self.spec = workload, spec
        self.kind = "port" if workload == "sdf_field" else "reference"
        if self.kind == "port":
            return
        if not refbind.host_available():
            raise RuntimeError("reference drivers (oracle/_ref) not built")
        self.r = refbind.RefScene(spec)
        cam = spec.camera
        if workload == "icospheres":
            self.w, self.h, self.spp = 16, 9, 1
            secs = self.r.render_cpu_parallel(cam, self.w, self.h, 1)[0]
            k = max(1, int((budget_s / max(secs, 1e-3)) ** 0.5))
            self.w, self.h = 16 * min(k, 12), 9 * min(k, 12)
        else:
            self.w, self.h = spec.width, spec.height
            secs = self.r.render_cpu_parallel(cam, self.w, self.h, 1)[0]
            self.spp = max(1, min(spec.spp, int(budget_s / max(secs, 1e-3))))

    def run(self):
        """One timed sample: (Mpaths/s, seconds, threads)."""
        if self.kind == "port":
            v, threads, self.desc = _port_sample(self.spec, self.spec.camera, 5.0)
            return v, None, threads
        secs, _, threads, _ = self.r.render_cpu_parallel(self.spec.camera, self.w, self.h, self.spp)
        return self.w * self.h * self.spp / secs / 1e6, secs, threads

    @property
    def sample(self) -> str:
        if self.kind == "port":
            return getattr(self, "desc", "FP64 oracle port on a pixel sample")
        what = ("the same camera at {}x{}".format(self.w, self.h) if self.workload == "icospheres"
                else "the {}x{} frame".format(self.w, self.h))
        return (f"RendererCPUParallel on {what} at {self.spp} spp ({self.w * self.h * self.spp} paths; FP64, linear "
                f"scan, depth 16, non-Lambert materials as Lambert)")


def cpu_baseline(workload: str, budget_s: float = 12.0):
    """The reference-arm CPU sample, once (rank 0, N = 1), for the line's cpu_baseline."""
    rs = RefCpuSample(workload, _ref_spec(workload), budget_s)
    v, secs, threads = rs.run()
    return {"value": v, "unit": "Mpaths/s", "cores": threads, "kind": rs.kind, "sample": rs.sample,
            "seconds": secs}


def run_reference(args):
    """The reference arm: the reference's own CPU renderer on a bounded sample per
    step of the same workload on all host threads (RefCpuSample), plus the
    reference's own CUDA renderer (renderAccKernel built for sm_100a from its
    sources) on the same frame where it can render the scene. Imports nothing
    from the rayon_b200 package: scenes come from oracle/workloads.py and the
    camera frame from the reference's CameraBase."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import refbind
    spec = _ref_spec(args.workload)
    desc = WORKLOADS[args.workload][2]
    w, h = spec.width, spec.height
    try:
        rs = RefCpuSample(args.workload, spec, 5.0)
    except RuntimeError as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return
    for _ in range(args.warmup if rs.kind == "reference" and args.workload != "icospheres" else 1):
        rs.run()
    vals, times, threads = [], [], 1
    for _ in range(args.steps if rs.kind == "reference" else max(1, min(args.steps, 3))):
        v1, secs, threads = rs.run()
        vals.append(v1)
        if secs is not None:
            times.append(secs)
    v = sum(vals) / len(vals)
    t = sum(times) / len(times) if times else None
    res = {
        "impl": "reference", "metric": METRIC if args.workload == "cornell" else f"Mpaths/s ({desc})",
        "value": v, "unit": "Mpaths/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3 if t else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{desc}; bounded sample per step: {rs.sample}", "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": "Mpaths/s", "cores": threads, "kind": rs.kind, "sample": rs.sample},
        "e2e": {"value": v, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.workload in ("cornell", "one_weekend"):
        try:
            res["reference_cuda"] = reference_cuda(spec)
        except Exception as e:  # noqa: BLE001
            res["reference_cuda"] = {"unavailable": f"{type(e).__name__}: {e}"}
    elif args.workload == "sdf_field":
        res["reference_cuda"] = {"unavailable": "the reference's GPU path skips SDF primitives "
                                                "(cuda_raytracer.cuh:372-373)"}
    else:
        res["reference_cuda"] = {"unavailable": "not timed: the reference builds this scene's BVH single-threaded "
                                                "(about 80 s for 5.2 M triangles)"}
    print(json.dumps(res))


WORKLOADS = {
    # name: (scene constructor, views per step, description); cornell is the
    # configuration the headline metric is quoted on
    "cornell": ("cornell", 1, "Cornell box 512x512, 256 spp, depth 16, 30 primitives, background 0"),
    "one_weekend": ("one_weekend", 1, "One-Weekend-style 488 spheres, 400x225, 32 spp, depth 10, depth of field"),
    "icospheres": ("icospheres", 1, "64 level-6 icospheres (5,242,880 triangles) + ground, 1920x1080, 64 spp, "
                                    "depth 8, GGX conductors"),
    "sdf_field": ("sdf_field", 16, "256 SDF primitives, smooth union k=0.2, 1280x720, 128 spp, depth 8, "
                                   "16 orbit views in one wavefront run"),
}
# engine per workload: the per-pixel / batched kernel, or the wavefront engine
# (whose separate field-march kernel is the faster one for SDF fields)
ENGINE = {"sdf_field": "wavefront"}
# wavefront queue: 0 = the path slots the autotuner chose for the scene
# (2 M to 16 M; 16 M slots take about 14 GB with the SDF march buffers)
WF_QUEUE = 0


def workload_spec(name: str, small: bool = False):
    from rayon_b200 import scenes
    ctor, views, desc = WORKLOADS[name]
    spec = getattr(scenes, ctor)()
    if small:  # profiling case: 16 spp, at most two views
        spec.spp = 16
        views = min(views, 2)
    return spec, views, desc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="rayon_b200")
    ap.add_argument("--workload", default="cornell", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the equal-RMSE and serving sections")
    ap.add_argument("--serving-jobs", type=int, default=2000,
                    help="jobs of the serving section's stream (default: the full specified stream of 2000 "
                         "Poisson arrivals at 50/s; about 9 minutes of plain and served runs)")
    ap.add_argument("--serving-by-scene", type=int, nargs="?", const=1, default=1,
                    help="serving section: also serve each scene's jobs alone (served/plain per scene; 0 = off)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the e2e repetitions (profiling runs)")
    ap.add_argument("--small", action="store_true",
                    help="profiling case for ncu: same frame at 16 spp (two views at most), no e2e/baselines")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.small:
        args.no_cpu_baseline = True
        args.no_e2e = True

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from rayon_b200 import lib, render
    spec, nviews, desc = workload_spec(args.workload, args.small)
    w, h, spp, depth = spec.width, spec.height, spec.spp, spec.depth
    cams = spec.views[:nviews] if nviews > 1 else [spec.camera]
    paths = w * h * spp * nviews
    sc = spec.to_scene()
    sc.build_bvh()
    frames = np.ascontiguousarray(np.stack([c.frame(w, h) for c in cams]), np.float64)
    fr = frames[0]
    # large scenes keep their built tree; the autotuner then tunes the launch only
    layout_kind = "autotune"

    def upload():
        if layout_kind == "autotune":
            return sc.upload(layout="autotune", tune_depth=depth, probe=(fr, w, h))
        return sc.upload()

    t_tune = time.perf_counter()
    ds = upload()
    tune_s = time.perf_counter() - t_tune
    layout = ds.layout
    frp = frames.ctypes.data_as(C.POINTER(C.c_double))
    render.set_globals(background=spec.background, dof=spec.dof)
    stream = torch.cuda.current_stream()
    sptr = C.c_void_p(stream.cuda_stream)
    npx = w * h
    engine = ENGINE.get(args.workload, "kernel")
    if engine == "wavefront":  # FP64 sums per view
        acc = torch.zeros((nviews, npx, 4), dtype=torch.float64, device="cuda")
    else:  # FP32 sums and Kahan terms per view
        acc = torch.zeros((nviews, 2, npx, 4), dtype=torch.float32, device="cuda")
    counters = torch.zeros(4, dtype=torch.int64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2

    def step(i, cnt=None):
        base = (rank * 1000003 + i) * spp % (1 << 30)
        cp = C.c_void_p(cnt.data_ptr()) if cnt is not None else None
        if engine == "wavefront":
            st = lib.rb_render_views_wavefront(ds.handle, nviews, w, h, frp, spp, base, depth,
                                               C.c_void_p(acc.data_ptr()), WF_QUEUE, cp, sptr)
        elif nviews > 1:
            st = lib.rb_render_views(ds.handle, nviews, w, h, frp, spp, base, depth, C.c_void_p(acc.data_ptr()),
                                     cp, sptr)
        else:
            st = lib.rb_render_accumulate(ds.handle, w, h, frp, spp, base, depth, C.c_void_p(acc.data_ptr()),
                                          C.c_void_p(acc.data_ptr() + npx * 16), cp, sptr)
        if st != 0:
            raise RuntimeError(render.lib.rb_last_error().decode())

    clk = ClockSampler(local).__enter__()
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    # segment / path counts of one step (for Mrays/s)
    counters.zero_()
    step(0, counters)
    torch.cuda.synchronize()
    segs, npaths, overflow = [int(x) for x in counters[:3].cpu()]

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = lib.rb_launch_count()
    evs = []
    # NVTX range "timed" lets a profiler select the timed launches only
    # (ncu --nvtx --nvtx-include "timed/"), past the layout probes and warm-up
    torch.cuda.nvtx.range_push("timed")
    lib.rb_kernel_timer_read(None, None)     # drop anything recorded before
    lib.rb_kernel_timer_enable(1)
    clk.mark(True)
    for i in range(args.steps):
        flush.fill_(float(i))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step(args.warmup + i)
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    clk.mark(False)
    lib.rb_kernel_timer_enable(0)
    k_ms, k_n = C.c_double(0.0), C.c_int64(0)
    lib.rb_kernel_timer_read(C.byref(k_ms), C.byref(k_n))
    clk.__exit__(None, None, None)
    torch.cuda.nvtx.range_pop()
    kernel_ms = k_ms.value / k_n.value if k_n.value else None   # per k_render launch, live
    launches = lib.rb_launch_count() - launches0
    ms = [a.elapsed_time(b) for a, b in evs]
    t_ms = sum(ms) / len(ms)
    if world > 1:
        tt = torch.tensor([t_ms], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t_ms = float(tt.item())
        torch.distributed.barrier()
    value = world * paths / (t_ms * 1e-3) / 1e6

    # ---- e2e through the public API with host buffers
    e2e = None
    mean_rad = None
    if not getattr(args, "no_e2e", False):
        torch.cuda.synchronize()
        e2e_times = []
        # the first repetition is a first call (staging buffers, the drop-in's
        # handles); the value is the median of the repetitions after it
        reps = 1 + max(1, min(5 if paths < (1 << 28) else 2, args.steps))
        parts = []
        for i in range(reps):
            t0 = time.perf_counter()
            ds2 = upload()  # layout decision cached per scene
            t_up = time.perf_counter()
            if args.workload == "cornell":
                # the drop-in call sequence of RayON's offline renderer
                img = render.render_dropin(ds2, fr, w, h, spp, depth, chunks=5)
                h2d = ds2.nbytes + npx * 12
                d2h = 5 * npx * 12
            elif engine == "wavefront":
                img = render.render_views_wavefront(ds2, list(frames), w, h, spp, depth, background=spec.background,
                                                    dof=spec.dof, queue_capacity=WF_QUEUE)
                h2d = ds2.nbytes + frames.nbytes
                d2h = nviews * npx * 32
            elif nviews > 1:
                img = render.render_views(ds2, list(frames), w, h, spp, depth, background=spec.background,
                                          dof=spec.dof)
                h2d = ds2.nbytes + frames.nbytes
                d2h = nviews * npx * 32
            else:
                img = render.render_accumulate(ds2, fr, w, h, spp, depth, background=spec.background,
                                               dof=spec.dof)
                h2d = ds2.nbytes
                d2h = npx * 32
            t_r = time.perf_counter()
            ds2.free()
            torch.cuda.synchronize()
            t_end = time.perf_counter()
            e2e_times.append(t_end - t0)
            parts.append({"upload_s": t_up - t0, "render_and_readback_s": t_r - t_up, "free_s": t_end - t_r})
        render.set_globals(background=spec.background, dof=spec.dof)
        steady = e2e_times[1:]
        e2e_t = statistics.median(steady)
        breakdown = parts[1 + steady.index(min(steady, key=lambda x: abs(x - e2e_t)))]
        if world > 1:  # the slowest rank bounds the job
            tt = torch.tensor([e2e_t], device="cuda")
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            e2e_t = float(tt.item())
        path = ("renderPixelsCUDAAccumulative x5 + scene upload (host float3 accumulation)"
                if args.workload == "cornell" else
                ("scene upload + rb_render_views_wavefront + accumulation readback" if engine == "wavefront" else
                 "scene upload + rb_render_views + accumulation readback" if nviews > 1 else
                 "scene upload + rb_render_accumulate + accumulation readback"))
        e2e = {"value": world * paths / e2e_t / 1e6, "unit": "Mpaths/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "seconds_per_step": e2e_t, "statistic": "median of repetitions 2..n",
               "best_mpaths_s": world * paths / min(steady) / 1e6, "path": path, "breakdown": breakdown,
               "all_seconds": e2e_times,
               "first_call": {"seconds": e2e_times[0], "breakdown": parts[0],
                              "layout_autotune_s": tune_s,
                              "note": "first repetition in this process after the timed steps; the layout "
                                      "autotune of the scene (layout_autotune_s) runs at its first upload"}}
        mean_rad = float(np.asarray(img).reshape(-1, 3).mean() / spp)

    split = sample_split_section(ds, fr, w, h, spp, depth, spec, engine, world) if world > 1 else None
    peaks, peaks_kind = measured_peaks()
    res = {
        "metric": f"Mpaths/s ({desc})" if args.workload != "cornell" else METRIC,
        "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "paths_per_step": paths,
                   "kernel": ("wavefront engine (k_wf_extend / k_wf_march / k_wf_shade over shared SoA queues "
                              "for all views)" if engine == "wavefront" else
                              "k_batch (persistent, one launch for all views)" if nviews > 1 else
                              "k_render (per-pixel, flattened sample x bounce loop)"),
                   "layout": layout, "tuning": ds.tuning,
                   "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{world}"},
        "mrays_per_s": world * segs / (t_ms * 1e-3) / 1e6,
        "segments_per_path": segs / max(npaths, 1),
        "stack_overflows": overflow,
        "gpu_launches": int(launches),
        "e2e": e2e,
    }
    if split is not None:
        res["sample_split"] = split
    clocks = clk.summary()
    res["clocks"] = clocks
    sm_mhz = clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    res["roofline"] = roofline(args.workload, peaks, peaks_kind, sm_mhz, t_ms, kernel_ms, segs, npaths, npx * nviews,
                               small=args.small)
    if not args.small:
        res["rmse_vs_oracle"] = config_error(args.workload, step, acc, engine, nviews, npx, spp, w, h)
    if args.workload == "icospheres" and not args.small:
        # the configuration asks for 8-bit quantised child bounds vs FP32 nodes
        res["node_layouts"] = node_layout_compare(sc, fr, w, h, spp, depth, step_ms=t_ms)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            res["cpu_baseline"] = cpu_baseline(args.workload)
        except Exception as e:  # noqa: BLE001
            res["cpu_baseline"] = {"unavailable": str(e)}
    res["mean_radiance"] = mean_rad
    if rank == 0 and world == 1 and args.workload == "cornell" and not args.small and not args.no_extras:
        for key, fn in (("equal_rmse", lambda: equal_rmse_section(t_ms, paths)),
                        ("serving", lambda: serving_section(args.serving_jobs, by_scene=args.serving_by_scene))):
            try:
                res[key] = fn()
            except Exception as e:  # noqa: BLE001
                res[key] = {"unavailable": f"{type(e).__name__}: {e}"}
    if rank == 0:
        print(json.dumps(res))
    if world > 1:
        torch.distributed.destroy_process_group()


def sample_split_section(ds, fr, w, h, spp, depth, spec, engine, world):
    """One frame of the workload split by samples over the ranks
    (multigpu.render_sample_split: rank r renders its sample range with the
    per-frame kernel, then one FP64 all-reduce over NCCL), timed with CUDA
    events between barriers, max over ranks: the strong-scaling form of the
    path next to the replicas of the main line. Rank 0 checks the reduced
    image against its own render of all the samples."""
    import torch
    import torch.distributed as dist

    from rayon_b200 import multigpu, render
    if engine != "kernel":
        return {"unavailable": "the sample split drives the per-frame kernel"}
    run = multigpu.gpu_range_renderer(ds, fr, w, h, depth, background=spec.background, dof=spec.dof)
    multigpu.render_sample_split(run, spp)          # warm-up (same collective steps on every rank)
    dist.barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    total = multigpu.render_sample_split(run, spp)
    b.record()
    torch.cuda.synchronize()
    t = torch.tensor([a.elapsed_time(b)], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    out = {"ms_per_frame": ms, "mpaths_s": w * h * spp / (ms * 1e-3) / 1e6, "ranks": world,
           "collective": "one FP64 all-reduce of the frame's sums (NCCL)"}
    if dist.get_rank() == 0:
        ref = render.render_accumulate(ds, fr, w, h, spp, depth, background=spec.background,
                                       dof=spec.dof).reshape(-1, 3)
        got = total.cpu().numpy()
        out["max_rel_diff_vs_one_gpu"] = float(np.max(np.abs(got - ref) / (1.0 + np.abs(ref))))
    return out


def node_layout_compare(sc, fr, w, h, spp, depth, step_ms):
    """One frame on each node layout of the same tree, uploaded as built with
    the class's default launch configuration (the same kernel, the same
    samples), median of 3 frames each: the binary tree with FP32 boxes (64 B
    nodes), the binary tree with 8-bit quantised boxes (32 B nodes) and the
    4-wide copy with FP32 boxes (128 B nodes, the default)."""
    import torch

    from rayon_b200 import lib
    out = {}
    frp = np.ascontiguousarray(fr, np.float64).ctypes.data_as(C.POINTER(C.c_double))
    acc = torch.zeros((w * h * 2, 4), dtype=torch.float32, device="cuda")
    for name, kw in (("binary_fp32", dict(wide=False)), ("binary_quantized", dict(quantized=True)),
                     ("wide_fp32", dict(wide=True))):
        d = sc.upload(**kw)
        args = (d.handle, w, h, frp, spp, 0, depth, C.c_void_p(acc.data_ptr()),
                C.c_void_p(acc.data_ptr() + w * h * 16), None, None)
        lib.rb_render_accumulate(*args)
        torch.cuda.synchronize()
        ms = []
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            lib.rb_render_accumulate(*args)
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        m = statistics.median(ms)
        out[name] = {"ms_per_frame": m, "mpaths_s": w * h * spp / (m * 1e-3) / 1e6, "device_bytes": d.nbytes}
        d.free()
    out["quantized_over_binary_time"] = out["binary_quantized"]["ms_per_frame"] / out["binary_fp32"]["ms_per_frame"]
    out["wide_over_binary_time"] = out["wide_fp32"]["ms_per_frame"] / out["binary_fp32"]["ms_per_frame"]
    out["tuned_timed_step_ms"] = step_ms
    return out


def reference_cuda(spec):
    """The reference's own CUDA renderer (renderAccKernel via its
    renderPixelsCUDAAccumulative, compiled for sm_100a from its sources) on
    the same frame: the scene through its SceneDescription, buildBVH and
    CudaSceneBuilder::buildGPUScene, the camera frame from its CameraBase, its
    setters for the workload (background, depth of field). Device: one
    device-resident call of all samples, timed with CUDA events (median of 5).
    e2e: RendererCUDA::render's loop (five calls with a host float3
    accumulation), wall clock, scene already resident; the scene build and
    upload are reported beside it."""
    from oracle import refbind
    if not refbind.cuda_available():
        return {"unavailable": "oracle/_ref/librayon_ref_cuda.so not built"}
    L = refbind.cuda()
    t0 = time.perf_counter()
    rs = refbind.RefCudaScene(spec)
    build_s = time.perf_counter() - t0
    dof = spec.dof or (0.1, 10.0)
    L.refc_set_globals(1.0, spec.background, 0.8, 1.5, int(spec.dof is not None), dof[0], dof[1])
    w, h = spec.width, spec.height
    fr = np.ascontiguousarray(refbind.camera_frame(spec.camera, w, h), np.float64)
    frp = fr.ctypes.data_as(C.POINTER(C.c_double))
    L.refc_render_device(rs.h, w, h, frp, 16, spec.depth, None)  # warm-up
    ms = [L.refc_render_device(rs.h, w, h, frp, spec.spp, spec.depth, None) for _ in range(5)]
    e2e = [L.refc_render(rs.h, w, h, frp, spec.spp, 5, spec.depth, None) for _ in range(3)]
    L.refc_set_globals(1.0, 1.0, 0.8, 1.5, 0, 0.1, 10.0)
    rs.free()
    if min(ms) <= 0 or min(e2e) <= 0:
        return {"unavailable": "the reference's CUDA render call failed (see its printed error)"}
    paths = w * h * spec.spp
    med, e2e_med = statistics.median(ms), statistics.median(e2e)
    return {"mpaths_s": paths / (med * 1e-3) / 1e6, "ms_per_frame": med, "ms_all": ms,
            "e2e_mpaths_s": paths / e2e_med / 1e6, "e2e_seconds_all": e2e, "scene_build_upload_s": build_s,
            "note": "reference renderAccKernel (sm_100a build of its sources, -maxrregcount 80, fast math); "
                    "e2e excludes its scene build and upload (scene_build_upload_s)"}


def serving_section(n_jobs: int = 2000, rate: float = 50.0, backlog: bool = False, by_scene: bool = True):
    """The serving mix: n_jobs Poisson arrivals at `rate` jobs/s (2000 in the
    specified stream) over the One-Weekend, Cornell, icosphere and SDF scenes,
    resolutions from {256^2, 512^2, 1280x720, 1920x1080}, spp log-uniform
    [16, 1024], orbit angle U[0, 2pi).

    plain: each job as its own per-frame launch, back to back, into one
    accumulation buffer allocated once, each launch timed with CUDA events
    (device seconds) and the loop on the wall clock; served: the batched
    serving loop with real-time arrivals (wall clock; device seconds from the
    server's own events); backlog (optional): the same jobs all queued at
    once. Ratios are wall/wall and device/device. by_scene: each scene's jobs
    of the mix served alone as a backlog, against the same jobs' plain
    launches (device time), so the gain is attributed scene by scene."""
    import torch

    from rayon_b200 import lib, render, scenes, serving
    t0 = time.time()
    specs = [scenes.one_weekend(), scenes.cornell(), scenes.icospheres(), scenes.sdf_field()]
    names = ["one_weekend", "cornell", "icospheres", "sdf_field"]
    dss = []
    for sp in specs:
        sc = sp.to_scene()
        sc.build_bvh()
        dss.append(sc.upload(layout="autotune", tune_depth=sp.depth))
    setup = time.time() - t0
    mix = scenes.serving_mix(n_jobs, rate=rate, n_scenes=len(specs))
    frames = [scenes.orbit(specs[j["scene"]].camera, j["angle"]).frame(j["width"], j["height"]) for j in mix]
    paths = sum(j["width"] * j["height"] * j["spp"] for j in mix)
    scene_paths = [sum(j["width"] * j["height"] * j["spp"] for j in mix if j["scene"] == i) for i in range(4)]
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))).__enter__()
    clocks = {}
    # plain per-job launches into one pre-allocated buffer
    maxpx = max(j["width"] * j["height"] for j in mix)
    acc = torch.zeros((2 * maxpx, 4), device="cuda")
    scene_dev = [0.0] * 4
    evs = []
    torch.cuda.synchronize()
    tp = time.time()
    clk.mark(True)
    for j, fr in zip(mix, frames):
        sp = specs[j["scene"]]
        n = j["width"] * j["height"]
        render.set_globals(background=sp.background, dof=sp.dof)
        acc[:2 * n].zero_()
        frc = np.ascontiguousarray(fr)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        lib.rb_render_accumulate(dss[j["scene"]].handle, j["width"], j["height"],
                                 frc.ctypes.data_as(C.POINTER(C.c_double)), j["spp"], 0, sp.depth,
                                 C.c_void_p(acc.data_ptr()), C.c_void_p(acc.data_ptr() + n * 16), None,
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
        b.record()
        evs.append((j["scene"], a, b))
    torch.cuda.synchronize()
    plain_wall = time.time() - tp
    clk.mark(False)
    for sidx, a, b in evs:
        scene_dev[sidx] += a.elapsed_time(b) * 1e-3
    plain_dev = sum(scene_dev)
    render.set_globals()
    del acc
    srv = serving.Server(paths_per_iteration=64 << 20, max_spp_per_iteration=64)
    ids = [srv.add_scene(ds) for ds in dss]
    reqs = [serving.job(ids[j["scene"]], fr, j["width"], j["height"], j["spp"], specs[j["scene"]].depth,
                        background=specs[j["scene"]].background, dof=specs[j["scene"]].dof, seed=k, arrival=j["t"])
            for k, (j, fr) in enumerate(zip(mix, frames))]
    tb = time.time()
    srv.run_trace(reqs, realtime=True)
    served_wall = time.time() - tb
    clk_t = (tb, time.time())
    st = srv.stats()
    srv.close()
    out_backlog = {}
    clk_b = None
    if backlog:  # the same jobs all queued at once: the loop's throughput without the arrival ramp
        srv = serving.Server(paths_per_iteration=64 << 20, max_spp_per_iteration=64)
        ids = [srv.add_scene(ds) for ds in dss]
        for r, j in zip(reqs, mix):
            r.scene = ids[j["scene"]]
            r.arrival_time = 0.0
        tb = time.time()
        srv.run_trace(reqs, realtime=False)
        wall_b = time.time() - tb
        clk_b = (tb, time.time())
        sb = srv.stats()
        srv.close()
        out_backlog = {"backlog_mpaths_s_wall": paths / wall_b / 1e6,
                       "backlog_mpaths_s_device": sb.paths / sb.device_seconds / 1e6 if sb.device_seconds else None}
    by_scene_out = {}
    if by_scene:
        for i, nm in enumerate(names):
            sel = [(r, j) for r, j in zip(reqs, mix) if j["scene"] == i]
            if not sel:
                continue
            srv = serving.Server(paths_per_iteration=64 << 20, max_spp_per_iteration=64)
            ids = [srv.add_scene(ds) for ds in dss]
            for r, j in sel:
                r.scene = ids[j["scene"]]
                r.arrival_time = 0.0
            tb = time.time()
            srv.run_trace([r for r, _ in sel], realtime=False)
            wall_s = time.time() - tb
            ss = srv.stats()
            srv.close()
            by_scene_out[nm] = {"jobs": len(sel),
                                "served_mpaths_s_device": scene_paths[i] / ss.device_seconds / 1e6
                                if ss.device_seconds else None,
                                "served_mpaths_s_wall": scene_paths[i] / wall_s / 1e6,
                                "plain_mpaths_s_device": scene_paths[i] / scene_dev[i] / 1e6 if scene_dev[i] else None,
                                "served_over_plain_device": scene_dev[i] / ss.device_seconds
                                if ss.device_seconds else None}
    clk.__exit__(None, None, None)
    path_csv = clk.path
    runs = [("plain", (clk.t0, clk.t1)), ("served", clk_t)] + ([("backlog", clk_b)] if clk_b else [])
    for name, (a, b) in runs:
        c = ClockSampler(clk.gpu)
        c.path, c.t0, c.t1 = path_csv, a, b
        clocks[name] = c.summary(keep=True)
    if path_csv and os.path.exists(path_csv):
        os.unlink(path_csv)
    for ds in dss:
        ds.free()
    served_dev = st.device_seconds
    res = {"jobs": n_jobs, "arrival_rate_per_s": rate, "paths": paths, "arrival_window_s": mix[-1]["t"],
           "offered_gpaths_per_s": paths / mix[-1]["t"] / 1e9,
           "plain_mpaths_s_wall": paths / plain_wall / 1e6, "plain_mpaths_s_device": paths / plain_dev / 1e6,
           "served_mpaths_s_wall": paths / served_wall / 1e6,
           "served_mpaths_s_device": st.paths / served_dev / 1e6 if served_dev else None,
           "served_over_plain_wall": plain_wall / served_wall,
           "served_over_plain_device": plain_dev / served_dev if served_dev else None,
           "p50_latency_s": st.p50_latency, "p99_latency_s": st.p99_latency, "mean_latency_s": st.mean_latency,
           "jobs_done": st.jobs_done, "jobs_rejected": st.jobs_rejected,
           "iterations": st.iterations, "peak_device_bytes": st.peak_device_bytes, "setup_s": setup,
           "plain_by_scene": {nm: {"path_share": scene_paths[i] / paths,
                                   "plain_mpaths_s_device": scene_paths[i] / scene_dev[i] / 1e6 if scene_dev[i] else None,
                                   "plain_time_share": scene_dev[i] / plain_dev}
                              for i, nm in enumerate(names)},
           "clocks": clocks,
           "note": "offered load exceeds one GPU's capacity, so latency is queue-dominated"}
    res.update(out_backlog)
    if by_scene_out:
        res["served_over_plain_by_scene"] = by_scene_out
    return res


def equal_rmse_section(full_ms_plain: float, full_paths: int):
    """Estimator efficiency at equal RMSE (Cornell box at 64x64): RMSE of
    64-spp renders with and without next-event estimation against the FP64
    oracle's converged image (4096 spp, NEE; the committed fixture
    tests/golden/oracle_cornell64.npz made by tests/golden/make_golden.py
    --oracle), combined with each estimator's Mpaths/s on the full 512x512
    frame."""
    import torch

    from rayon_b200 import lib, render, scenes
    spec = scenes.cornell(width=64, height=64)
    sc = spec.to_scene()
    sc.build_bvh()
    ds = sc.upload(layout="autotune", tune_depth=spec.depth)
    fr = spec.camera.frame(64, 64)
    fx = np.load(ROOT / "tests" / "golden" / "oracle_cornell64.npz")
    ref = fx["mean"].astype(np.float64)
    oracle_s = float(fx["seconds"])
    out = {}
    for nee in (False, True):
        errs = []
        for k in range(4):
            img = render.render_accumulate(ds, fr, 64, 64, 64, spec.depth, background=0.0, nee=nee,
                                           sample_base=64 * k) / 64
            errs.append(np.sqrt(((img - ref) ** 2).mean()))
        out["rmse_nee" if nee else "rmse_plain"] = float(np.mean(errs))
    ds.free()
    # NEE throughput on the full frame
    big = scenes.cornell()
    scb = big.to_scene()
    scb.build_bvh()
    dsb = scb.upload(layout="autotune", tune_depth=big.depth)
    frb = big.camera.frame(big.width, big.height)
    with render.options(nee=True):
        render.set_globals(background=0.0)
        acc = torch.zeros((big.width * big.height * 2, 4), device="cuda")
        frc = np.ascontiguousarray(frb)
        args = (dsb.handle, big.width, big.height, frc.ctypes.data_as(C.POINTER(C.c_double)), big.spp, 0, big.depth,
                C.c_void_p(acc.data_ptr()), C.c_void_p(acc.data_ptr() + big.width * big.height * 16), None, None)
        lib.rb_render_accumulate(*args)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        lib.rb_render_accumulate(*args)
        b.record()
        torch.cuda.synchronize()
        ms_nee = a.elapsed_time(b)
        render.set_globals()
    dsb.free()
    mp_plain = full_paths / (full_ms_plain * 1e-3) / 1e6
    mp_nee = full_paths / (ms_nee * 1e-3) / 1e6
    out.update({"mpaths_s_plain": mp_plain, "mpaths_s_nee": mp_nee, "oracle_seconds": oracle_s,
                "equal_rmse_speedup_nee": (mp_nee / mp_plain) * (out["rmse_plain"] / out["rmse_nee"]) ** 2,
                "note": "RMSE of 64-spp 64x64 renders vs FP64 oracle at 4096 spp; speedup = throughput ratio x "
                        "variance ratio (paths needed for equal RMSE)"})
    return out


if __name__ == "__main__":
    main()
