"""Render calls over the C-ABI. Device buffers are torch CUDA tensors (plumbing
only); every kernel is the native library's."""
from __future__ import annotations

import ctypes as C
import threading
from contextlib import contextmanager

import numpy as np

from ._native import RenderOpts, check, lib

DEFAULT_SEED = 0x5EED


def _torch():
    import torch
    return torch


def _stream_ptr():
    torch = _torch()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


_staging = threading.local()


def _pinned_like(t):
    """A pinned host tensor of t's shape and dtype, kept per thread and reused:
    the copy back runs at full DMA speed and touches no fresh pages."""
    torch = _torch()
    cache = getattr(_staging, "bufs", None)
    if cache is None:
        cache = _staging.bufs = {}
    key = (tuple(t.shape), t.dtype)
    buf = cache.get(key)
    if buf is None:
        if len(cache) > 8:
            cache.clear()
        buf = cache[key] = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    return buf


def set_globals(light: float = 1.0, background: float = 1.0, fuzz: float = 0.8, glass_ior: float = 1.5,
                dof: tuple | None = None) -> None:
    """The reference's shading setters (renderer_cuda_device.cuh:36-50); defaults = its __constant__ values."""
    lib.setLightIntensity(light)
    lib.setBackgroundIntensity(background)
    lib.setMetalFuzziness(fuzz)
    lib.setGlassRefractionIndex(glass_ior)
    lib.setDOFEnabled(dof is not None)
    if dof is not None:
        lib.setDOFAperture(float(dof[0]))
        lib.setDOFFocusDistance(float(dof[1]))
    else:
        lib.setDOFAperture(0.1)
        lib.setDOFFocusDistance(10.0)


def get_opts() -> RenderOpts:
    o = RenderOpts()
    lib.rb_get_render_opts(C.byref(o))
    return o


_SCHEDULES = {"auto": 0, "grid": 1, "fetch": 2}


def set_opts(nee: bool | None = None, kahan: bool | None = None, seed: int | None = None,
             block: tuple | None = None, blocks_per_sm: int | None = None, slices: int | None = None,
             schedule: str | None = None) -> None:
    """Render options of the per-pixel kernel (rb_render_opts). blocks_per_sm:
    register budget in resident 256-thread blocks (0 = tuned); slices: sample
    slices per pixel (0 = automatic); schedule: "grid", "fetch" (persistent
    warps taking 8x4-pixel tiles from a counter) or "auto" (the scene's tuned
    schedule)."""
    o = get_opts()
    if blocks_per_sm is not None:
        o.reserved[0] = int(blocks_per_sm)
    if slices is not None:
        o.reserved[1] = int(slices)
    if schedule is not None:
        o.reserved[2] = _SCHEDULES[schedule]
    if nee is not None:
        o.nee = int(nee)
    if kahan is not None:
        o.kahan = int(kahan)
    if seed is not None:
        o.seed = int(seed)
    if block is not None:
        o.block_x, o.block_y = int(block[0]), int(block[1])
    lib.rb_set_render_opts(C.byref(o))


@contextmanager
def options(**kw):
    old = get_opts()
    try:
        set_opts(**kw)
        yield
    finally:
        lib.rb_set_render_opts(C.byref(old))


def primary_hits(ds, frame: np.ndarray, w: int, h: int, return_t: bool = False):
    torch = _torch()
    ids = torch.empty(w * h, dtype=torch.int32, device="cuda")
    t = torch.empty(w * h, dtype=torch.float32, device="cuda")
    fr = np.ascontiguousarray(frame, np.float64)
    check(lib.rb_primary_hits(ds.handle, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(ids.data_ptr()),
                              C.c_void_p(t.data_ptr()), _stream_ptr()), "rb_primary_hits")
    torch.cuda.synchronize()
    ids_np = ids.cpu().numpy().reshape(h, w)
    if return_t:
        return ids_np, t.cpu().numpy().reshape(h, w)
    return ids_np


def render_accumulate(ds, frame, w: int, h: int, spp: int, depth: int, background: float = 1.0,
                      dof: tuple | None = None, nee: bool = False, sample_base: int = 0, kahan: bool = True,
                      seed: int = DEFAULT_SEED, light: float = 1.0, fuzz: float = 0.8, glass_ior: float = 1.5,
                      counters: bool = False):
    """Per-pixel radiance sums (h, w, 3) float64 of samples [sample_base, sample_base + spp)."""
    torch = _torch()
    set_globals(light=light, background=background, fuzz=fuzz, glass_ior=glass_ior, dof=dof)
    # sums, then Kahan compensations, in one allocation (one fill, one copy back)
    buf = torch.zeros((2 if kahan else 1, w * h, 4), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(4, dtype=torch.int64, device="cuda") if counters else None
    fr = np.ascontiguousarray(frame, np.float64)
    with options(nee=nee, seed=seed):
        check(lib.rb_render_accumulate(ds.handle, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)), spp, sample_base,
                                       depth, C.c_void_p(buf[0].data_ptr()),
                                       C.c_void_p(buf[1].data_ptr()) if kahan else None,
                                       C.c_void_p(cnt.data_ptr()) if cnt is not None else None, _stream_ptr()),
              "rb_render_accumulate")
        stage = _pinned_like(buf)
        stage.copy_(buf, non_blocking=True)
        torch.cuda.current_stream().synchronize()
    host = stage.numpy()
    img = np.empty((w * h, 3), np.float64)
    if kahan:  # Kahan: true sum = sum - compensation, subtracted in FP64
        np.subtract(host[0, :, :3], host[1, :, :3], out=img, dtype=np.float64)
    else:
        img[:] = host[0, :, :3]
    img = img.reshape(h, w, 3)
    set_globals()
    if counters:
        return img, cnt.cpu().numpy()
    return img


def render_wavefront(ds, frame, w: int, h: int, spp: int, depth: int, background: float = 1.0,
                     dof: tuple | None = None, nee: bool = False, sample_base: int = 0, seed: int = DEFAULT_SEED,
                     queue_capacity: int = 0, counters: bool = False):
    """Per-pixel radiance sums (h, w, 3) float64 from the wavefront engine (FP64 accumulation)."""
    torch = _torch()
    set_globals(background=background, dof=dof)
    acc = torch.zeros((w * h, 4), dtype=torch.float64, device="cuda")
    cnt = torch.zeros(4, dtype=torch.int64, device="cuda")
    fr = np.ascontiguousarray(frame, np.float64)
    with options(nee=nee, seed=seed):
        check(lib.rb_render_wavefront(ds.handle, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)), spp, sample_base,
                                      depth, C.c_void_p(acc.data_ptr()), int(queue_capacity),
                                      C.c_void_p(cnt.data_ptr()), _stream_ptr()), "rb_render_wavefront")
        torch.cuda.synchronize()
    set_globals()
    img = acc[:, :3].cpu().numpy().reshape(h, w, 3)
    return (img, cnt.cpu().numpy()) if counters else img


def render_views(ds, frames, w: int, h: int, spp: int, depth: int, background: float = 1.0,
                 dof: tuple | None = None, nee: bool = False, sample_base: int = 0, seed: int = DEFAULT_SEED,
                 counters: bool = False):
    """Per-view radiance sums (n_views, h, w, 3) float64 of several camera frames
    rendered in one persistent launch (rb_render_views); view v uses salt v."""
    torch = _torch()
    fr = np.ascontiguousarray(np.stack([np.asarray(f, np.float64) for f in frames]))
    n = fr.shape[0]
    set_globals(background=background, dof=dof)
    acc = torch.zeros((n, 2, w * h, 4), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(4, dtype=torch.int64, device="cuda")
    with options(nee=nee, seed=seed):
        check(lib.rb_render_views(ds.handle, n, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)), spp, sample_base,
                                  depth, C.c_void_p(acc.data_ptr()), C.c_void_p(cnt.data_ptr()), _stream_ptr()),
              "rb_render_views")
        torch.cuda.synchronize()
    set_globals()
    img = (acc[:, 0, :, :3].double() - acc[:, 1, :, :3].double()).cpu().numpy().reshape(n, h, w, 3)
    return (img, cnt.cpu().numpy()) if counters else img


def render_views_wavefront(ds, frames, w: int, h: int, spp: int, depth: int, background: float = 1.0,
                           dof: tuple | None = None, nee: bool = False, sample_base: int = 0,
                           seed: int = DEFAULT_SEED, queue_capacity: int = 0, counters: bool = False):
    """Per-view radiance sums (n_views, h, w, 3) float64 of several camera frames
    rendered by one wavefront run over all views (rb_render_views_wavefront)."""
    torch = _torch()
    fr = np.ascontiguousarray(np.stack([np.asarray(f, np.float64) for f in frames]))
    n = fr.shape[0]
    set_globals(background=background, dof=dof)
    acc = torch.zeros((n, w * h, 4), dtype=torch.float64, device="cuda")
    cnt = torch.zeros(4, dtype=torch.int64, device="cuda")
    with options(nee=nee, seed=seed):
        check(lib.rb_render_views_wavefront(ds.handle, n, w, h, fr.ctypes.data_as(C.POINTER(C.c_double)), spp,
                                            sample_base, depth, C.c_void_p(acc.data_ptr()), int(queue_capacity),
                                            C.c_void_p(cnt.data_ptr()), _stream_ptr()), "rb_render_views_wavefront")
        torch.cuda.synchronize()
    set_globals()
    img = acc[:, :, :3].cpu().numpy().reshape(n, h, w, 3)
    return (img, cnt.cpu().numpy()) if counters else img


def render_dropin(ds, frame, w: int, h: int, spp: int, depth: int, chunks: int = 5):
    """RendererCUDA::render's loop (renderer_cuda_host.hpp:35-58) through the drop-in
    entry point with a host float3 accumulation buffer. Returns (h, w, 3) float32 sums."""
    accum = np.zeros(w * h * 3, np.float32)
    rng = C.c_void_p(None)
    dacc = C.c_void_p(None)
    per = max(1, spp // chunks)
    done = 0
    fr = frame
    while done < spp:
        add = min(per, spp - done)
        done += add
        n = lib.renderPixelsCUDAAccumulative(None, accum.ctypes.data_as(C.POINTER(C.c_float)), ds.handle, w, h,
                                             fr[0], fr[1], fr[2], fr[3], fr[4], fr[5], fr[6], fr[7], fr[8], fr[9],
                                             fr[10], fr[11], add, done, depth, C.byref(rng), C.byref(dacc), fr[12],
                                             fr[13], fr[14], fr[15], fr[16], fr[17], None, 32, 0.01)
        if n != w * h * add:
            raise RuntimeError(f"renderPixelsCUDAAccumulative failed: {lib.rb_last_error().decode()}")
    lib.freeDeviceRandomStates(rng)
    lib.freeDeviceAccumBuffer(dacc)
    return accum.reshape(h, w, 3)
