// The per-pixel progressive kernel (k_render) and its launch helpers,
// templated on the node layout its traversal reads (RB_NODES_BINARY /
// RB_NODES_WIDE). rb_render.cu instantiates the binary-tree kernels and
// rb_render_wide.cu the wide-tree ones, so the two sets compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "rb_internal.hpp"
#include "rb_path.cuh"

namespace rb {
using namespace rbd;

// One pixel's sample slice z of nz: the pixel's samples of the slice back to
// back in one flattened loop (one path segment per iteration). Adds the
// thread's segments and paths to segs and paths.
template <bool NEE, int MS, int NODES>
__device__ __forceinline__ void render_pixel_slice(const SceneView &S, const Globals &G, const FrameF &P, int x, int y,
                                                   int z, int nz, int2 *smem, int tid, int threads,
                                                   float4 *__restrict__ acc, float4 *__restrict__ comp,
                                                   float4 *__restrict__ part, int *__restrict__ counts,
                                                   unsigned long long *__restrict__ counters,
                                                   unsigned long long &segs, unsigned long long &paths) {
  const bool inside = x < P.width && y < P.height;
  const int pix = inside ? y * P.width + x : 0;
  int have = 0;
  bool work = inside;
  if (work && counts) {
    have = counts[pix];
    if (have < 0) work = false;  // converged (sign bit, render_acc_kernel.cu:165-170)
  }
  if (work) {
    Stack st;
    stack_init(st, smem, tid, threads, S.short_stack);
    uint32_t ovf = 0;
    // sample slice z of nz (small frames split their samples so that the
    // launch fills the GPU): slice 0 adds into the pixel's sums, the others
    // leave partial sums in part for k_fold_slices
    const int s_begin = (int)((long long)P.samples * z / nz);
    const int s_end = (int)((long long)P.samples * (z + 1) / nz);
    float sx = 0.f, sy = 0.f, sz = 0.f;
    float cx = 0.f, cy = 0.f, cz = 0.f;
    if (z == 0) {
      const float4 a0 = acc[pix];
      sx = a0.x; sy = a0.y; sz = a0.z;
      if (comp) {
        const float4 c0 = comp[pix];
        cx = c0.x; cy = c0.y; cz = c0.z;
      }
    }
    float lum_before = 0.0f;
    if (counts && have > 0) {
      const float inv = 1.0f / (float)have;
      lum_before = 0.299f * sx * inv + 0.587f * sy * inv + 0.114f * sz * inv;
    }
    int s = s_begin, bounce = 0;
    bool alive = false;
    Ray ray;
    f3 thr(1.f, 1.f, 1.f), L(0.f, 0.f, 0.f);
    uint32_t key = 0;
    float prev_pdf = 0.0f;
    const int nsamples = P.max_depth > 0 ? s_end : 0;  // depth 0: no bounce, black (ray_color's empty loop)
    while (true) {
      if (!alive) {
        if (s >= nsamples) break;
        key = rb_path_key(P.seed, P.salt, (uint32_t)pix, (uint32_t)(P.sample_base + s));
        ++s;
        ray = camera_ray(P, G, x, y, key);
        thr = f3(1.f, 1.f, 1.f);
        L = f3(0.f, 0.f, 0.f);
        bounce = 0;
        prev_pdf = 0.0f;
        alive = true;
      }
      ++segs;
      if (path_segment<NEE, MS, NODES>(S, G, st, ovf, ray, thr, L, bounce, prev_pdf, key, P.max_depth)) {
        if (comp) {
          kahan_add(sx, cx, L.x);
          kahan_add(sy, cy, L.y);
          kahan_add(sz, cz, L.z);
        } else {
          sx += L.x; sy += L.y; sz += L.z;
        }
        alive = false;
      }
    }
    if (z == 0) {
      acc[pix] = make_float4(sx, sy, sz, 0.0f);
      if (comp) comp[pix] = make_float4(cx, cy, cz, 0.0f);
    } else {
      part[(size_t)(z - 1) * P.width * P.height + pix] = make_float4(sx - cx, sy - cy, sz - cz, 0.0f);
    }
    if (counts) {  // convergence test (render_acc_kernel.cu:241-271); counts are never split
      const int nc = have + P.samples;
      if (nc >= P.min_adaptive) {
        const float inv = 1.0f / (float)nc;
        const float lum_after = 0.299f * sx * inv + 0.587f * sy * inv + 0.114f * sz * inv;
        const float rel = fabsf(lum_after - lum_before) / fmaxf(lum_after, 0.001f);
        counts[pix] = rel < P.adaptive_threshold ? -nc : nc;
      } else {
        counts[pix] = nc;
      }
    }
    if (counters && ovf) atomicAdd(counters + 2, (unsigned long long)ovf);
    paths += (unsigned long long)(s_end - s_begin);
  }
}

// Per-pixel progressive kernel: one thread owns one pixel for the launch and
// runs its samples back to back in a single flattened loop (one path segment
// per iteration), so a lane whose path ended starts its next sample at once
// instead of idling until the warp's longest path finishes.
//
// Two schedules of the same work. Grid mode (fetch == nullptr): one thread per
// pixel of a 2-D grid of bx x by blocks, sample slice blockIdx.z of gridDim.z.
// Fetch mode: a persistent grid of 1-D blocks sized to the SMs' resident
// capacity; each warp takes work items (a tile of 8 x 4 pixels in one sample
// slice of `nslices`) from the counter *fetch until they run out, so a warp
// whose tile finished early starts the next one instead of idling until its
// block's other warps and the launch's last wave finish. Items run slice-major,
// then tile rows, so concurrent warps work on neighbouring tiles. A pixel's
// slice is computed by one thread in sample order either way: the sums are the
// same bit for bit.
#define RB_TILE_W 8
#define RB_TILE_H 4
template <bool NEE, int MS, int MINB, int NODES>
__global__ void __launch_bounds__(256, MINB) k_render(const RB_GRID_CONST SceneView S,
                                                      const RB_GRID_CONST Globals G,
                                                      const RB_GRID_CONST FrameF P, float4 *__restrict__ acc,
                                                float4 *__restrict__ comp, float4 *__restrict__ part,
                                                int *__restrict__ counts, unsigned long long *__restrict__ counters,
                                                int *__restrict__ fetch, int nslices) {
  extern __shared__ int2 smem[];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int threads = blockDim.x * blockDim.y;
  const int lane = tid & 31;
  const int tiles_x = (P.width + RB_TILE_W - 1) / RB_TILE_W;
  const int tiles = tiles_x * ((P.height + RB_TILE_H - 1) / RB_TILE_H);
  const long long items = fetch ? (long long)tiles * nslices : 0;
  unsigned long long segs = 0, paths = 0;
  for (;;) {
    int x, y, z, nz;
    if (fetch) {
      int it = 0;
      if (lane == 0) it = atomicAdd(fetch, 1);
      it = __shfl_sync(0xffffffffu, it, 0);
      if (it >= items) break;
      z = it / tiles;
      const int tile = it - z * tiles;
      const int ty = tile / tiles_x;
      x = (tile - ty * tiles_x) * RB_TILE_W + (lane & (RB_TILE_W - 1));
      y = ty * RB_TILE_H + lane / RB_TILE_W;
      nz = nslices;
    } else {
      x = blockIdx.x * blockDim.x + threadIdx.x;
      y = blockIdx.y * blockDim.y + threadIdx.y;
      z = blockIdx.z;
      nz = gridDim.z;
    }
    render_pixel_slice<NEE, MS, NODES>(S, G, P, x, y, z, nz, smem, tid, threads, acc, comp, part, counts, counters, segs,
                                paths);
    if (!fetch) break;
  }
  if (counters) {
    // warp-aggregated segment and path counts
    for (int o = 16; o > 0; o >>= 1) {
      segs += __shfl_down_sync(0xffffffffu, segs, o);
      paths += __shfl_down_sync(0xffffffffu, paths, o);
    }
    if (lane == 0) {
      atomicAdd(counters, segs);
      atomicAdd(counters + 1, paths);
    }
  }
}

// One k_render launch of register budget minb (1-4 resident 256-thread blocks
// per SM).
template <bool NEE, int MS, int NODES>
static void launch_k_render(int minb, dim3 grd, dim3 blk, size_t sm, cudaStream_t st, const SceneView &S,
                            const Globals &G, const FrameF &P, float4 *acc, float4 *comp, float4 *part, int *counts,
                            unsigned long long *counters, int *fetch, int nslices) {
  switch (minb) {
    case 1: k_render<NEE, MS, 1, NODES><<<grd, blk, sm, st>>>(S, G, P, acc, comp, part, counts, counters, fetch, nslices); break;
    case 3: k_render<NEE, MS, 3, NODES><<<grd, blk, sm, st>>>(S, G, P, acc, comp, part, counts, counters, fetch, nslices); break;
    case 4: k_render<NEE, MS, 4, NODES><<<grd, blk, sm, st>>>(S, G, P, acc, comp, part, counts, counters, fetch, nslices); break;
    default: k_render<NEE, MS, 2, NODES><<<grd, blk, sm, st>>>(S, G, P, acc, comp, part, counts, counters, fetch, nslices); break;
  }
}

// Resident blocks per SM of that kernel at `threads` threads and `sm` bytes
// of dynamic shared memory (the persistent grid of fetch mode).
template <bool NEE, int MS, int NODES>
static int k_render_resident_blocks(int minb, int threads, size_t sm) {
  int n = 0;
  cudaError_t e;
  switch (minb) {
    case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_render<NEE, MS, 1, NODES>, threads, sm); break;
    case 3: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_render<NEE, MS, 3, NODES>, threads, sm); break;
    case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_render<NEE, MS, 4, NODES>, threads, sm); break;
    default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_render<NEE, MS, 2, NODES>, threads, sm); break;
  }
  return e == cudaSuccess && n > 0 ? n : 1;
}

// Dispatch over (NEE, material class) for one node layout: a launch, or (with
// launch == false) the resident-block query.
template <int NODES>
static int k_render_dispatch(bool launch, bool nee, int ms, int minb, dim3 grd, dim3 blk, size_t sm, cudaStream_t st,
                             const SceneView &S, const Globals &G, const FrameF &P, float4 *acc, float4 *comp,
                             float4 *part, int *counts, unsigned long long *counters, int *fetch, int nslices) {
#define RB_K(NEE_, MS_)                                                                                     \
  do {                                                                                                      \
    if (!launch) return k_render_resident_blocks<NEE_, MS_, NODES>(minb, (int)(blk.x * blk.y * blk.z), sm);   \
    launch_k_render<NEE_, MS_, NODES>(minb, grd, blk, sm, st, S, G, P, acc, comp, part, counts, counters, fetch, \
                                      nslices);                                                            \
    return 0;                                                                                               \
  } while (0)
  if (nee) {
    if (ms == RB_MS_DIFFUSE) RB_K(true, RB_MS_DIFFUSE);
    if (ms == RB_MS_CLASSIC) RB_K(true, RB_MS_CLASSIC);
    if (ms == RB_MS_FULL) RB_K(true, RB_MS_FULL);
    RB_K(true, RB_MS_SDF);
  }
  if (ms == RB_MS_DIFFUSE) RB_K(false, RB_MS_DIFFUSE);
  if (ms == RB_MS_CLASSIC) RB_K(false, RB_MS_CLASSIC);
  if (ms == RB_MS_FULL) RB_K(false, RB_MS_FULL);
  RB_K(false, RB_MS_SDF);
#undef RB_K
}

// The wide-tree instances (rb_render_wide.cu).
int k_render_dispatch_wide(bool launch, bool nee, int ms, int minb, dim3 grd, dim3 blk, size_t sm, cudaStream_t st,
                           const SceneView &S, const Globals &G, const FrameF &P, float4 *acc, float4 *comp,
                           float4 *part, int *counts, unsigned long long *counters, int *fetch, int nslices);

}  // namespace rb
