"""Python handle on the native serving loop (rb_server_*): continuous batching
of render jobs over resident scenes. The loop itself is C++ (rb_batch.cu)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import JobRequest, JobStatus, ServerOpts, ServerStats, check, lib


def job(scene: int, frame, width: int, height: int, spp: int, depth: int, background: float = 1.0,
        dof: tuple | None = None, nee: bool = False, seed: int = 0, fp64: bool = False, arrival: float = 0.0,
        light: float = 1.0, fuzz: float = 0.8, glass_ior: float = 1.5, converge: tuple | None = None) -> JobRequest:
    """converge = (threshold, min_spp, fraction): complete the job early once
    that fraction of its pixels change by less than the threshold per iteration."""
    r = JobRequest()
    lib.rb_job_default(C.byref(r))
    r.scene, r.width, r.height, r.spp, r.max_depth = scene, width, height, spp, depth
    r.frame[:] = [float(v) for v in frame]
    r.background_intensity, r.light_intensity, r.metal_fuzziness, r.glass_ior = background, light, fuzz, glass_ior
    if dof is not None:
        r.dof_enabled, r.dof_aperture, r.dof_focus = 1, float(dof[0]), float(dof[1])
    r.nee, r.seed, r.fp64_accum, r.arrival_time = int(nee), int(seed), int(fp64), float(arrival)
    if converge is not None:
        r.converge_threshold, r.converge_min_spp, r.converge_fraction = (float(converge[0]), int(converge[1]),
                                                                         float(converge[2]))
    return r


class Server:
    def __init__(self, budget_bytes: int | None = None, max_jobs: int | None = None, paths_per_iteration=None,
                 max_spp_per_iteration=None, use_graph: bool = True, frames_every: int = 0, occupancy: int = 0,
                 wavefront_field: bool = True, target_iteration_ms: float = 0.0, stream=None,
                 per_frame_classes: int | None = None):
        o = ServerOpts()
        lib.rb_server_default_opts(C.byref(o))
        if budget_bytes is not None:
            o.memory_budget_bytes = int(budget_bytes)
        if max_jobs is not None:
            o.max_active_jobs = int(max_jobs)
        if paths_per_iteration is not None:
            o.paths_per_iteration = int(paths_per_iteration)
        if max_spp_per_iteration is not None:
            o.max_spp_per_iteration = int(max_spp_per_iteration)
        o.use_graph, o.frames_every, o.occupancy = int(use_graph), int(frames_every), int(occupancy)
        o.wavefront_field = int(wavefront_field)
        o.target_iteration_ms = float(target_iteration_ms)
        if per_frame_classes is not None:
            o.per_frame_classes = int(per_frame_classes)
        self.h = lib.rb_server_create(C.byref(o), stream)
        if not self.h:
            raise RuntimeError(lib.rb_last_error().decode())

    def add_scene(self, ds) -> int:
        return check(lib.rb_server_add_scene(self.h, ds.handle), "add_scene")

    def submit(self, req: JobRequest) -> int:
        return check(lib.rb_server_submit(self.h, C.byref(req)), "submit")

    def step(self) -> int:
        return check(lib.rb_server_step(self.h), "step")

    def drain(self) -> None:
        while self.step() > 0:
            pass

    def status(self, jid: int) -> JobStatus:
        s = JobStatus()
        check(lib.rb_server_job_status(self.h, jid, C.byref(s)), "status")
        return s

    def fetch(self, jid: int, width: int, height: int, frame: bool = False):
        rgb = np.zeros(width * height * 3, np.float32)
        fr = np.zeros(width * height * 4, np.uint8) if frame else None
        check(lib.rb_server_fetch(self.h, jid, rgb.ctypes.data_as(C.POINTER(C.c_float)),
                                  fr.ctypes.data_as(C.POINTER(C.c_uint8)) if fr is not None else None), "fetch")
        out = rgb.reshape(height, width, 3)
        return (out, fr.reshape(height, width, 4)) if frame else out

    def release(self, jid: int) -> None:
        check(lib.rb_server_release(self.h, jid), "release")

    def run_trace(self, reqs: list, realtime: bool = True, keep: bool = False) -> np.ndarray:
        arr = (JobRequest * len(reqs))(*reqs)
        lat = np.zeros(len(reqs), np.float64)
        check(lib.rb_server_run_trace(self.h, arr, len(reqs), int(realtime), int(keep),
                                      lat.ctypes.data_as(C.POINTER(C.c_double))), "run_trace")
        return lat

    def stats(self) -> ServerStats:
        s = ServerStats()
        check(lib.rb_server_get_stats(self.h, C.byref(s)), "stats")
        return s

    def close(self) -> None:
        if self.h:
            lib.rb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
