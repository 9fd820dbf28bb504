// Wavefront engine: the path tracer split into queue-connected kernels.
//
// Path state lives in structure-of-arrays queues of 16-byte elements (every
// access is one 128-bit load or store, coalesced across the warp):
//   o      float4 (origin xyz, prev. diffuse pdf)     d    float4 (direction xyz, -)
//   thr    float4 (throughput xyz, -)                 L    float4 (radiance xyz, -)
//   meta   int4   (pixel, sample, bounce, path key)   hit  float4 (t, prim, -, -)
//   sn     float4 (SDF field normal xyz, material)    (written only on field hits)
// One iteration is these launches over the live paths of queue A:
//   extend: trace each ray to its closest hit (traversal only: few registers,
//           high occupancy for latency hiding);
//   shade:  surface, material scatter, emission, next-event estimation,
//           Russian roulette; a path that ends adds its radiance to the
//           pixel (FP64 atomics: order-independent sums). Survivors are
//           written compacted into queue B, each block's range claimed by
//           its last warp to finish;
//   regen:  the free slots of queue B take new camera paths for the next
//           work items (path regeneration; a one-thread plan launch, then
//           one thread per new path).
// Scenes with a smooth SDF field add a launch between extend and shade:
// extend only collects each ray's field candidates (a 256-bit set of SDF
// primitives, or sorted 16-byte records of index and window [t0, t1]) and
// appends the ray to a march list; march is a persistent kernel whose lanes
// each take a ray from the list, advance it one sphere-tracing step per pass
// and take the next ray as soon as theirs finishes, so a warp does not wait
// for its slowest ray (a march takes from one to hundreds of steps).
// The queues then swap. Work items are sample-major (consecutive lanes take
// consecutive pixels of the same sample) so primary rays of a warp are
// coherent and the accumulation atomics of a warp hit distinct pixels. The
// same counter-based sample streams as the per-frame kernel are used, so the
// two engines agree path for path. Iterations are recorded once into a CUDA
// graph (8 iterations per graph launch, ping-ponging the queues) and replayed
// until the live count reaches zero.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "rb_path.cuh"

namespace rb {

extern std::atomic<unsigned long long> g_launches;
DeviceScene *lookup_scene(const void *handle);

struct WfQueue {
  float4 *o, *d, *thr, *L, *hit, *sn;
  int4 *meta;
};

struct WfCtl {
  unsigned long long next_path;   // next work item to generate
  unsigned long long total_paths; // pixels * samples
  int count[2];                   // live paths in queue 0 / 1
  unsigned long long segments;
  unsigned long long paths_done;
  unsigned long long overflow;
  int march_count;                // rays appended to the march list this iteration
  unsigned int march_next;        // next march-list entry to take
  unsigned long long march_steps;
  unsigned long long regen_item;  // k_wf_regen: the first new work item,
  int regen_slot;                 // its slot,
  int regen_n;                    // and how many
};

struct WfParams {
  SceneView S;
  const WfJob *jobs;  // device table of njobs jobs
  int njobs;
  WfCtl *ctl;
  // smooth SDF field (null otherwise): candidate records of queue slot k at
  // cand[i * cap + k], i < ncand[k]; list = slots to march
  int4 *cand;
  int *ncand;
  int *list;
  int cap;
};

// The engine's shared counters (queue fill, march list, work items, segment
// and path counts) are one address each, and the L2 serialises atomics on one
// address: one atomic per warp in a launch of 16 M slots is 512 K atomics on
// each. The extend and shade kernels therefore claim once per block, by the
// block's last warp to finish: each warp stages what it produced in shared
// memory and leaves, and a shared count of finished warps (after a block
// fence) tells the last one, which claims the block's range with one atomic
// and copies the staged entries out. No warp waits at a barrier for the
// others. New camera paths are not emitted by the shade kernel: a separate
// launch fills the output queue's free slots with consecutive work items
// (k_wf_regen_plan, k_wf_regen).

// List entries a march warp claims at once when it runs short (0: one claim
// per refill of exactly the lanes that need a ray).
#ifndef WF_MARCH_CHUNK
#define WF_MARCH_CHUNK 32
#endif

// True for the block's last warp to arrive (call once per warp, after the
// warp's shared-memory writes; `done` is a zeroed shared counter).
__device__ __forceinline__ bool wf_last_warp(unsigned *done) {
  __syncwarp();
  __threadfence_block();
  unsigned d = 0;
  if ((threadIdx.x & 31) == 0) d = atomicAdd(done, 1u);
  d = __shfl_sync(0xffffffffu, d, 0);
  const bool last = d == ((blockDim.x + 31u) >> 5) - 1u;
  if (last) __threadfence_block();
  return last;
}

__device__ __forceinline__ bool wf_marches(const WfParams &W) {
  return W.cand != nullptr && W.S.sdf_k > 0.0f && W.S.num_sdf > 0;
}

__device__ __forceinline__ int wf_find_job(const WfParams &W, unsigned long long item) {
  int lo = 0, hi = W.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&W.jobs[mid].item_begin) <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Generates the camera ray of work item `item` into queue slot `k`; the
// path's meta record carries (pixel, job, bounce, path key).
__device__ __forceinline__ void wf_emit_camera(const WfParams &W, const WfQueue &q, int k, unsigned long long item) {
  const int j = wf_find_job(W, item);
  const WfJob &J = W.jobs[j];
  const unsigned long long local = item - J.item_begin;
  const int npix = J.P.width * J.P.height;
  const int pix = (int)(local % (unsigned long long)npix);
  const int sample = (int)(local / (unsigned long long)npix);
  const uint32_t key = rb_path_key(J.P.seed, J.P.salt, (uint32_t)pix, (uint32_t)(J.P.sample_base + sample));
  const Ray r = camera_ray(J.P, J.G, pix % J.P.width, pix / J.P.width, key);
  q.o[k] = make_float4(r.o.x, r.o.y, r.o.z, 0.0f);
  q.d[k] = make_float4(r.d.x, r.d.y, r.d.z, 0.0f);
  q.thr[k] = make_float4(1.f, 1.f, 1.f, 0.f);
  q.L[k] = make_float4(0.f, 0.f, 0.f, 0.f);
  q.meta[k] = make_int4(pix, j, 0, (int)key);
}

// Initial fill of queue `qi` with min(capacity, total) fresh paths.
__global__ void k_wf_fill(const RB_GRID_CONST WfParams W, const RB_GRID_CONST WfQueue q, int qi,
                          int capacity) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long total = W.ctl->total_paths;
  const unsigned long long n = total < (unsigned long long)capacity ? total : (unsigned long long)capacity;
  if ((unsigned long long)k < n) wf_emit_camera(W, q, k, (unsigned long long)k);
  if (k == 0) {
    W.ctl->count[qi] = (int)n;
    W.ctl->next_path = n;
  }
}

// Four resident blocks per SM (64 registers): +7 % on the SDF field over
// three at 72 (the traversal waits on its node loads). The shade kernel stays
// at two (128 registers): three and four spill and ran 2-6 % slower.
#ifndef WF_EXTEND_MINB
#define WF_EXTEND_MINB 4
#endif
// Candidate sets of the smooth SDF field: RB_SDF_MASK_BITS-bit masks (tables
// of at most that many primitives; rows 0 and 1 of the candidate buffer hold
// words 0-3 and 4-7) or, for larger tables, sorted window records.
#ifndef WF_SDF_MASK
#define WF_SDF_MASK 1
#endif
template <int MS, bool MASK>
__global__ void __launch_bounds__(256, WF_EXTEND_MINB) k_wf_extend(const RB_GRID_CONST WfParams W,
                                                                   const RB_GRID_CONST WfQueue q, int qi) {
  extern __shared__ int2 smem[];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  __shared__ int s_marched[256];      // the block's marching slots (blocks of at most 256 threads)
  __shared__ unsigned s_nm, s_done;  // staged slots, finished warps
  if (MS >= RB_MS_SDF) {
    if (threadIdx.x == 0) {
      s_nm = 0u;
      s_done = 0u;
    }
    __syncthreads();  // at the start every warp arrives together
  }
  const bool valid = k < W.ctl->count[qi];
  bool march = false;
  if (valid) {
    Stack st;
    stack_init(st, smem, threadIdx.x, blockDim.x, W.S.short_stack);
    uint32_t ovf = 0;
    const float4 o = q.o[k], d = q.d[k];
    Ray r;
    r.o = f3(o.x, o.y, o.z);
    r.d = f3(d.x, d.y, d.z);
    if (MS >= RB_MS_SDF && MASK && wf_marches(W)) {
      // traversal only: the field is marched by k_wf_march; the crossed
      // primitives are kept as a bit set (index order, no per-ray arrays)
      SdfMask cand;
      cand.clear();
      const HitInfo h = trace_bvh<false, MS, RB_SPEC_TRAVERSAL, SdfMask>(W.S, r, 0.001f, FLT_MAX, st, ovf, &cand);
      q.hit[k] = make_float4(h.t, __int_as_float(h.prim), 0.f, 0.f);
      if (cand.any()) {
        W.cand[k] = make_int4((int)cand.w[0], (int)cand.w[1], (int)cand.w[2], (int)cand.w[3]);
        W.cand[(size_t)W.cap + k] = make_int4((int)cand.w[4], (int)cand.w[5], (int)cand.w[6], (int)cand.w[7]);
        march = true;
      }
    } else if (MS >= RB_MS_SDF && wf_marches(W)) {
      // traversal only: the field is marched by k_wf_march
      SdfCand cand;
      cand.n = 0;
      const HitInfo h = trace_bvh<false, MS, RB_SPEC_TRAVERSAL>(W.S, r, 0.001f, FLT_MAX, st, ovf, &cand);
      q.hit[k] = make_float4(h.t, __int_as_float(h.prim), 0.f, 0.f);
      if (cand.n > 0) {
        sdf_sort_cand(cand);
        for (int i = 0; i < cand.n; ++i)
          W.cand[(size_t)i * W.cap + k] =
              make_int4(cand.idx[i], __float_as_int(cand.t0[i]), __float_as_int(cand.t1[i]), 0);
        W.ncand[k] = cand.n;
        march = true;
      }
    } else {
      const HitInfo h = trace<false, MS, RB_SPEC_TRAVERSAL>(W.S, r, 0.001f, FLT_MAX, st, ovf);
      q.hit[k] = make_float4(h.t, __int_as_float(h.prim), 0.f, 0.f);
      if (MS >= RB_MS_SDF && h.prim == -2)
        q.sn[k] = make_float4(h.sdf_n.x, h.sdf_n.y, h.sdf_n.z, __int_as_float(h.sdf_mat));
    }
    if (ovf) atomicAdd(&W.ctl->overflow, (unsigned long long)ovf);
  }
  if (MS >= RB_MS_SDF) {
    // append the marching rays to the list: each warp stages its slots in
    // shared memory and leaves; the block's last warp to finish claims the
    // block's range with one atomic and copies the slots out (no warp waits
    // for the others)
    const unsigned m = __ballot_sync(0xffffffffu, march);
    if (m) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(&s_nm, (unsigned)__popc(m));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (march) s_marched[base + __popc(m & ((1u << lane) - 1u))] = k;
    }
    if (wf_last_warp(&s_done)) {
      const unsigned n = *static_cast<volatile unsigned *>(&s_nm);
      int at = 0;
      if (lane == 0 && n) at = atomicAdd(&W.ctl->march_count, (int)n);
      at = __shfl_sync(0xffffffffu, at, 0);
      for (unsigned i = lane; i < n; i += 32) W.list[at + (int)i] = static_cast<volatile int *>(s_marched)[i];
    }
  }
}

// Field of the candidates of queue slot `slot` (the same operations, in the
// same order, as sdf_field_eval over an in-register candidate list). The first
// WF_CAND_REG candidate records are passed in registers (loaded once per ray),
// the rest are read from the slot's records.
#define WF_CAND_REG 4
__device__ __forceinline__ int4 wf_cand(const WfParams &W, const int4 (&cr)[WF_CAND_REG], int slot, int i) {
  int4 e = cr[0];
#pragma unroll
  for (int k = 1; k < WF_CAND_REG; ++k)
    if (i == k) e = cr[k];
  return i < WF_CAND_REG ? e : __ldg(W.cand + (size_t)i * W.cap + slot);
}

// Two passes so that a warp's lanes evaluate together: first each lane marks,
// in index order, its candidates whose window holds t (and the next window
// entry beyond t); then the lanes fold their k-th marked candidate at the
// same time, k = 0, 1, ... (the fold order per lane is still index order).
//
// The mark pass: the candidates whose window holds t, the next entry beyond
// t, and the earliest exit among the held windows. The set stays the same
// while t < next and t <= that exit (t never decreases along a march), so the
// march recomputes it only when t leaves that range.
__device__ __forceinline__ void wf_mark(const WfParams &W, const int4 (&cr)[WF_CAND_REG], int slot, int n, float t,
                                        uint32_t &active, float &next, float &exit) {
  uint32_t a = 0;
  float nx = RB_SDF_FAR, ex = RB_SDF_FAR;
  for (int i = 0; i < n; ++i) {
    const int4 e = wf_cand(W, cr, slot, i);
    const float t0 = __int_as_float(e.y), t1 = __int_as_float(e.z);
    if (t0 > t) nx = fminf(nx, t0);
    else if (t <= t1) {
      a |= 1u << i;
      ex = fminf(ex, t1);
    }
  }
  active = a;
  next = nx;
  exit = ex;
}

// The fold pass over the marked candidates: the field at p (RB_SDF_FAR when
// none is marked); `lone` is the candidate code when exactly one is marked.
__device__ __forceinline__ float wf_fold(const SceneView &S, const WfParams &W, const float4 *tab, int slot,
                                         const int4 (&cr)[WF_CAND_REG], uint32_t active, const f3 &p, int *nearest,
                                         int &lone) {
  const bool single = active != 0u && (active & (active - 1u)) == 0u;
  lone = -1;
  float F = RB_SDF_FAR, best = RB_SDF_FAR;
  bool first = true;
  while (active) {
    const int i = __ffs(active) - 1;
    active &= active - 1;
    const int code = wf_cand(W, cr, slot, i).x;
    if (single) lone = code;
    const int id = code >> 1;
    const float d = tab ? sdf_eval_words(tab[5 * id], tab[5 * id + 1], tab[5 * id + 2], tab[5 * id + 3],
                                         tab[5 * id + 4], p)
                        : sdf_eval_at(S.sdf, id, p);
    if (nearest && d < best) {
      best = d;
      *nearest = id;
    }
    F = first ? d : smin_poly(F, d, S.sdf_k);
    first = false;
  }
  return F;
}

// --- candidate sets as bit masks (tables of at most RB_SDF_MASK_BITS primitives)
// The window of table entry i along the ray: its k-inflated bounding sphere
// (centre in word 0, radius in word 4), the same operations as the extend
// kernel's collection test. false when the ray misses the sphere.
__device__ __forceinline__ bool wf_window(const float4 *tab, int i, const Ray &r, float aa, float &t0, float &t1) {
  const float4 w0 = tab[5 * i], w4 = tab[5 * i + 4];
  const f3 oc = r.o - f3(w0.x, w0.y, w0.z);
  const float hb = dot(oc, r.d), cc = dot(oc, oc) - w4.z * w4.z;
  const float disc = hb * hb - aa * cc;
  if (disc < 0.0f) return false;
  const float sq = sqrtf(disc);
  t0 = (-hb - sq) / aa;
  t1 = (-hb + sq) / aa;
  return true;
}

#define WF_MARK_REG 4
// Marks, in index order, the candidates whose window holds t: the first
// WF_MARK_REG of them in mid[] (registers), their total in *count; also the
// next window entry beyond t and the earliest exit among the held windows.
__device__ __forceinline__ void wf_mark_mask(const float4 *tab, const uint32_t (&cm)[RB_SDF_MASK_WORDS], const Ray &r,
                                             float t, int (&mid)[WF_MARK_REG], int &count, float &next, float &exit) {
  const float aa = dot(r.d, r.d);
  float nx = RB_SDF_FAR, ex = RB_SDF_FAR;
  int c = 0;
#pragma unroll
  for (int w = 0; w < RB_SDF_MASK_WORDS; ++w) {
    uint32_t m = cm[w];
    while (m) {
      const int i = 32 * w + __ffs(m) - 1;
      m &= m - 1;
      float t0, t1;
      if (!wf_window(tab, i, r, aa, t0, t1)) continue;
      if (t0 > t) {
        nx = fminf(nx, t0);
      } else if (t <= t1) {
#pragma unroll
        for (int k = 0; k < WF_MARK_REG; ++k)
          if (k == c) mid[k] = i;
        ++c;
        ex = fminf(ex, t1);
      }
    }
  }
  count = c;
  next = nx;
  exit = ex;
}

// One marked candidate folded into the field at p.
__device__ __forceinline__ void wf_fold_one(const SceneView &S, const float4 *tab, int i, const f3 &p, float &F,
                                            bool &first, float &best, int *nearest) {
  const float d = sdf_eval_words(tab[5 * i], tab[5 * i + 1], tab[5 * i + 2], tab[5 * i + 3], tab[5 * i + 4], p);
  if (nearest && d < best) {
    best = d;
    *nearest = i;
  }
  F = first ? d : smin_poly(F, d, S.sdf_k);
  first = false;
}

// The field at p over the marked candidates (RB_SDF_FAR when none): the
// lanes fold their k-th marked candidate together; a ray holding more than
// WF_MARK_REG windows at t finds the rest again from its candidate mask
// (indices above mid[WF_MARK_REG - 1], window test at t). `lone` is the
// candidate code (index << 1 | convex) when exactly one window holds t.
__device__ __forceinline__ float wf_fold_mask(const SceneView &S, const float4 *tab,
                                              const uint32_t (&cm)[RB_SDF_MASK_WORDS], const Ray &r, float t,
                                              const int (&mid)[WF_MARK_REG], int count, const f3 &p, int *nearest,
                                              int &lone) {
  float F = RB_SDF_FAR, best = RB_SDF_FAR;
  bool first = true;
  lone = -1;
  const int nreg = count < WF_MARK_REG ? count : WF_MARK_REG;
#pragma unroll
  for (int k = 0; k < WF_MARK_REG; ++k)
    if (k < nreg) wf_fold_one(S, tab, mid[k], p, F, first, best, nearest);
  if (count == 1) lone = (mid[0] << 1) | (__float_as_int(tab[5 * mid[0] + 4].w) & 1);
  if (count > WF_MARK_REG) {  // rare: more windows hold t than the registers keep
    const float aa = dot(r.d, r.d);
    const int after = mid[WF_MARK_REG - 1];
#pragma unroll
    for (int w = 0; w < RB_SDF_MASK_WORDS; ++w) {
      uint32_t m = cm[w];
      while (m) {
        const int i = 32 * w + __ffs(m) - 1;
        m &= m - 1;
        float t0, t1;
        if (i > after && wf_window(tab, i, r, aa, t0, t1) && t0 <= t && t <= t1)
          wf_fold_one(S, tab, i, p, F, first, best, nearest);
      }
    }
  }
  return F;
}

// Persistent field march over the march list. Every pass, each busy lane
// evaluates the field exactly once, whatever its phase, so the warp's lanes
// evaluate in lockstep: escape (stepping out of the eps shell, up to 8
// passes), march (one sphere-tracing step of sdf_field_march's loop, its
// convex skip included) and, at a hit, the six central differences of the
// normal (one per pass). The
// nearest primitive (the hit's material) is tracked in every march
// evaluation, which at the hit is the evaluation at the hit point itself. A
// lane whose ray finishes (hit, windows left behind, closest primitive hit
// passed, steps used up) takes the next ray from the list (one atomic per
// warp). A field hit replaces the ray's hit record.
enum : int { WF_ESCAPE = 0, WF_MARCH = 1, WF_NORMAL = 2 };

// Four resident 256-thread blocks per SM (64 registers, a few bytes spilled):
// the march is latency-bound, and 50 % occupancy beat 37.5 % by 7 % on the
// SDF field.
#ifndef WF_MARCH_MINB
#define WF_MARCH_MINB 4
#endif
template <int MS, bool MASK>
__global__ void __launch_bounds__(256, WF_MARCH_MINB) k_wf_march(WfParams W, WfQueue q, int stage_table) {
  extern __shared__ float4 s_tab[];
  const int lane = threadIdx.x & 31;
  const SceneView &S = W.S;
  // stage the SDF table in shared memory when it fits (stage_table != 0)
  if (stage_table) {
    const float4 *g = reinterpret_cast<const float4 *>(S.sdf);
    for (int i = threadIdx.x; i < 5 * S.num_sdf; i += blockDim.x) s_tab[i] = __ldg(g + i);
    __syncthreads();
  }
  const float4 *tab = stage_table ? s_tab : nullptr;
  const unsigned total = (unsigned)W.ctl->march_count;
  const float e = RB_SDF_NORMAL_EPS;
  int slot = 0, n = 0, steps = 0, phase = WF_ESCAPE, sub = 0, nearest = 0, prev = -1;
  float prev_d = 0.f;
  // the lane's marked window set and the t range it holds for (wf_mark)
  uint32_t marked = 0;
  float mark_next = -1.f, mark_exit = -1.f;
  int4 cr[WF_CAND_REG];
#pragma unroll
  for (int i = 0; i < WF_CAND_REG; ++i) cr[i] = make_int4(0, 0, 0, 0);
  // MASK: the ray's candidate mask and its marked windows (first WF_MARK_REG in registers)
  uint32_t cm[RB_SDF_MASK_WORDS];
  int mid[WF_MARK_REG];
  int mcount = 0;
#pragma unroll
  for (int i = 0; i < RB_SDF_MASK_WORDS; ++i) cm[i] = 0u;
#pragma unroll
  for (int i = 0; i < WF_MARK_REG; ++i) mid[i] = 0;
  float t = 0.f, tmax = 0.f, sgn = 1.f, inv_len = 1.f;
  f3 p(0.f, 0.f, 0.f), g(0.f, 0.f, 0.f);
  Ray r;
  r.o = r.d = f3(0.f, 0.f, 0.f);
  bool busy = false, drained = false;
  unsigned long long passes = 0;
  unsigned cl_next = 0, cl_end = 0;  // the warp's claimed list range (the same in every lane)
  while (true) {
    const bool need = !busy && !drained;
    const unsigned mask = __ballot_sync(0xffffffffu, need);
    if (mask) {
      const int leader = __ffs(mask) - 1;
      const unsigned want = (unsigned)__popc(mask), rank = (unsigned)__popc(mask & ((1u << lane) - 1u));
      unsigned idx_base = 0;  // this lane's list entry is idx_base + rank (below) or in the new range
#if WF_MARCH_CHUNK
      // the warp keeps a claimed range [cl_next, cl_end) of list entries and
      // takes a new range of at least WF_MARCH_CHUNK when it runs short (one
      // atomic per range instead of one per refill)
      const unsigned avail = cl_end - cl_next;
      unsigned nb = 0, take = 0;
      if (avail < want) {
        take = want - avail > WF_MARCH_CHUNK ? want - avail : WF_MARCH_CHUNK;
        if (lane == leader) nb = atomicAdd(&W.ctl->march_next, take);
        nb = __shfl_sync(0xffffffffu, nb, leader);
      }
      idx_base = rank < avail ? cl_next : nb - avail;
      if (avail >= want) {
        cl_next += want;
      } else {
        cl_next = nb + (want - avail);
        cl_end = nb + take;
      }
#else
      if (lane == leader) idx_base = atomicAdd(&W.ctl->march_next, want);
      idx_base = __shfl_sync(0xffffffffu, idx_base, leader);
#endif
      if (need) {
        const unsigned idx = idx_base + rank;
        if (idx < total) {
          slot = W.list[idx];
          if constexpr (MASK) {
            const int4 a = __ldg(W.cand + slot), b = __ldg(W.cand + (size_t)W.cap + slot);
            cm[0] = (uint32_t)a.x; cm[1] = (uint32_t)a.y; cm[2] = (uint32_t)a.z; cm[3] = (uint32_t)a.w;
            cm[4] = (uint32_t)b.x; cm[5] = (uint32_t)b.y; cm[6] = (uint32_t)b.z; cm[7] = (uint32_t)b.w;
          } else {
            n = W.ncand[slot];
#pragma unroll
            for (int i = 0; i < WF_CAND_REG; ++i)
              if (i < n) cr[i] = __ldg(W.cand + (size_t)i * W.cap + slot);
          }
          const float4 o = q.o[slot], d = q.d[slot];
          r.o = f3(o.x, o.y, o.z);
          r.d = f3(d.x, d.y, d.z);
          tmax = q.hit[slot].x;
          inv_len = 1.0f / r.d.length();
          t = 0.001f;
          phase = WF_ESCAPE;
          sub = 0;
          steps = 0;
          prev = -1;
          mark_next = -1.f;  // mark again for the new ray
          busy = true;
        } else {
          drained = true;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, busy) == 0) break;
    if (!busy) continue;
    ++passes;
    // the one evaluation of this pass
    f3 pe;
    if (phase == WF_NORMAL) {
      const float off = (sub & 1) ? -e : e;
      pe = p + f3(sub < 2 ? off : 0.f, (sub >> 1) == 1 ? off : 0.f, sub >= 4 ? off : 0.f);
    } else {
      pe = r.at(t);
    }
    int near, lone;
    float raw;
    if constexpr (MASK) {
      if (!(t < mark_next && t <= mark_exit)) wf_mark_mask(tab, cm, r, t, mid, mcount, mark_next, mark_exit);
      near = mid[0];
      raw = wf_fold_mask(S, tab, cm, r, t, mid, mcount, pe, phase == WF_NORMAL ? nullptr : &near, lone);
    } else {
      if (!(t < mark_next && t <= mark_exit)) wf_mark(W, cr, slot, n, t, marked, mark_next, mark_exit);
      near = cr[0].x >> 1;
      raw = wf_fold(S, W, tab, slot, cr, marked, pe, phase == WF_NORMAL ? nullptr : &near, lone);
    }
    const float next = mark_next;
    bool finished = false;
    if (phase == WF_NORMAL) {
      if (sub & 1) {
        if (sub == 1) g.x = g.x - raw;
        else if (sub == 3) g.y = g.y - raw;
        else g.z = g.z - raw;
      } else {
        if (sub == 0) g.x = raw;
        else if (sub == 2) g.y = raw;
        else g.z = raw;
      }
      if (++sub == 6) {
        const float gl = g.length();
        const f3 nv = gl > 0.0f ? g / gl : f3(0.0f, 1.0f, 0.0f);
        q.hit[slot] = make_float4(t, __int_as_float(-2), 0.f, 0.f);
        q.sn[slot] = make_float4(nv.x, nv.y, nv.z, __int_as_float(S.sdf[nearest].material));
        finished = true;
      }
    } else {
      if (phase == WF_ESCAPE) {
        if (fabsf(raw) < 2.0f * S.sdf_eps && sub < 8) {
          t += 2.0f * S.sdf_eps * inv_len;
          ++sub;
        } else {
          sgn = raw < 0.0f ? -1.0f : 1.0f;
          phase = WF_MARCH;  // and this evaluation is the first march step's
        }
      }
      if (phase == WF_MARCH) {
        if (raw == RB_SDF_FAR) {  // between windows: jump to the next entry
          if (next == RB_SDF_FAR || next > tmax) finished = true;
          else t = next;
          prev = -1;
        } else {
          const float F = sgn * raw;
          if (F < S.sdf_eps) {
            if (t <= tmax) {
              p = pe;
              nearest = near;
              phase = WF_NORMAL;
              sub = 0;
            } else {
              finished = true;
            }
          } else {
            const int one = (sgn > 0.0f && lone >= 0 && (lone & 1)) ? lone : -1;
            if (one >= 0 && one == prev && raw > RB_SDF_SKIP_GROWTH * prev_d) {  // convex skip
              if (next == RB_SDF_FAR || next > tmax) finished = true;
              else t = next;
              prev = -1;
            } else {
              prev = one;
              prev_d = raw;
              t = fminf(t + F * inv_len, next);
              if (t > tmax) finished = true;
            }
          }
        }
        if (!finished && phase == WF_MARCH && ++steps >= S.sdf_steps) finished = true;
      }
    }
    if (finished) busy = false;
  }
  for (int o2 = 16; o2 > 0; o2 >>= 1) passes += __shfl_down_sync(0xffffffffu, passes, o2);
  if (lane == 0 && passes) atomicAdd(&W.ctl->march_steps, passes);
}

// Threads per shade block (a block claims once for all its warps, so its
// warps wait for one another at the claim).
#ifndef WF_SHADE_THREADS
#define WF_SHADE_THREADS 256
#endif
#ifndef WF_SHADE_MINB
#define WF_SHADE_MINB 2
#endif
template <int MS, bool NEE>
__global__ void __launch_bounds__(256, WF_SHADE_MINB) k_wf_shade(WfParams W, WfQueue in, WfQueue out, int qi) {
  extern __shared__ int2 smem[];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int n_in = W.ctl->count[qi];
  __shared__ float4 s_rec[5 * WF_SHADE_THREADS];  // the block's surviving paths (o, d, thr, L, meta)
  __shared__ unsigned s_nout, s_nend, s_nlive, s_done;
  if (threadIdx.x == 0) {
    s_nout = 0u;
    s_nend = 0u;
    s_nlive = 0u;
    s_done = 0u;
  }
  __syncthreads();  // at the start every warp arrives together
  bool have_out = false;
  // outgoing path, held in registers until the warp's range is reserved
  float4 no = make_float4(0, 0, 0, 0), nd = no, nthr = no, nL = no;
  int4 nmeta = make_int4(0, 0, 0, 0);
  bool regenerate = false;
  if (k < n_in) {
    Stack st;
    stack_init(st, smem, threadIdx.x, blockDim.x, W.S.short_stack);
    uint32_t ovf = 0;
    const float4 o = in.o[k], d = in.d[k], th = in.thr[k], Lv = in.L[k], hv = in.hit[k];
    const int4 m = in.meta[k];
    const Globals G = W.jobs[m.y].G;
    const int max_depth = W.jobs[m.y].P.max_depth;
    Ray ray;
    ray.o = f3(o.x, o.y, o.z);
    ray.d = f3(d.x, d.y, d.z);
    f3 thr(th.x, th.y, th.z), L(Lv.x, Lv.y, Lv.z);
    float prev_pdf = o.w;
    int bounce = m.z;
    const uint32_t key = (uint32_t)m.w;
    HitInfo h;
    h.t = hv.x;
    h.prim = __float_as_int(hv.y);
    if (MS >= RB_MS_SDF && h.prim == -2) {
      const float4 s = in.sn[k];
      h.sdf_n = f3(s.x, s.y, s.z);
      h.sdf_mat = __float_as_int(s.w);
    }
    // shade with the precomputed hit (path_segment's body after its trace)
    bool ended = false;
    if (h.prim == -1) {
      if (G.background_intensity != 0.0f) L = L + thr * sky(ray.d) * G.background_intensity;
      ended = true;
    } else {
      const Surface sf = surface<MS>(W.S, ray, h);
      if (!sf.visible && bounce == 0) {
        ray.o = sf.p + ray.d * 0.01f;
        ended = ++bounce >= max_depth;
      } else if (sf.mat >= W.S.num_mats) {
        ended = true;
      } else {
        const DevMaterial &mt = W.S.mats[sf.mat];
        const ScatterOut so = scatter<MS>(G, mt, sf, ray, key, bounce);
        if (so.emit.length_squared() > 0.0f) {
          float wgt = 1.0f;
          if (NEE && G.nee && prev_pdf > 0.0f && mt.kind == L_LIGHT && W.S.num_lights > 0) {
            const float dl = h.t * ray.d.length();
            const float cl = fabsf(dot(sf.n, normalize(ray.d)));
            const float pl = cl > 0.0f ? dl * dl / (cl * W.S.light_area) : 0.0f;
            wgt = mis2(prev_pdf, pl);
          }
          L = L + thr * so.emit * wgt;
        }
        if (!so.scattered) {
          ended = true;
        } else {
          if (NEE && G.nee) {
            prev_pdf = 0.0f;
            if (mt.kind == L_LAMBERTIAN && bounce + 1 < max_depth && W.S.num_lights > 0) {
              LightSample ls;
              const uint32_t dl = rb_vdim(bounce, RB_SLOT_LIGHT);
              if (sample_light(W.S, G, rb_draw(key, dl), rb_draw(key, dl + 1), rb_draw(key, dl + 2), ls)) {
                const f3 dv = ls.p - so.ray.o;
                const float d2 = dv.length_squared();
                const float dist = sqrtf(d2);
                const f3 wi = dv / dist;
                const float cs = dot(normalize(sf.n), wi);
                const float cl = fabsf(dot(ls.n, wi));
                if (cs > 0.0f && cl > 0.0f) {
                  Ray sr;
                  sr.o = so.ray.o;
                  sr.d = wi;
                  const HitInfo sh = trace<true, MS, RB_SPEC_TRAVERSAL>(W.S, sr, 0.001f, dist * (1.0f - 1e-4f), st, ovf);
                  if (sh.prim == -1) {
                    const float pl = d2 / (cl * W.S.light_area);
                    const float pb = cs * (1.0f / RB_PI);
                    L = L + thr * so.att * ls.Le * (cs * (1.0f / RB_PI) * mis2(pl, pb) / pl);
                  }
                }
              }
              prev_pdf = so.pdf;
            }
          }
          thr = thr * so.att;
          if (bounce > 0) {
            const float sp = fminf(fmaxf(thr.x, fmaxf(thr.y, thr.z)), 0.95f);
            if (rb_draw(key, rb_vdim(bounce, RB_SLOT_RR)) > sp) ended = true;
            else thr = thr / sp;
          }
          if (!ended) {
            ray = so.ray;
            ended = ++bounce >= max_depth;
          }
        }
      }
    }
    if (ended) {
      double *a = W.jobs[m.y].acc + 4 * (size_t)m.x;
      atomicAdd(a, (double)L.x);
      atomicAdd(a + 1, (double)L.y);
      atomicAdd(a + 2, (double)L.z);
      regenerate = true;
    } else {
      have_out = true;
      no = make_float4(ray.o.x, ray.o.y, ray.o.z, prev_pdf);
      nd = make_float4(ray.d.x, ray.d.y, ray.d.z, 0.0f);
      nthr = make_float4(thr.x, thr.y, thr.z, 0.0f);
      nL = make_float4(L.x, L.y, L.z, 0.0f);
      nmeta = make_int4(m.x, m.y, bounce, m.w);
    }
    if (ovf) atomicAdd(&W.ctl->overflow, (unsigned long long)ovf);
  }
  // Survivors are compacted into the output queue by the block's last warp
  // (each warp stages its surviving paths in shared memory and leaves); the
  // ended paths are only counted: k_wf_regen fills the free slots with new
  // camera paths after this launch.
  const unsigned mo = __ballot_sync(0xffffffffu, have_out), me = __ballot_sync(0xffffffffu, regenerate);
  const unsigned ml = __ballot_sync(0xffffffffu, k < n_in);
  unsigned off = 0;
  if (lane == 0) {
    if (mo) off = atomicAdd(&s_nout, (unsigned)__popc(mo));
    if (me) atomicAdd(&s_nend, (unsigned)__popc(me));
    if (ml) atomicAdd(&s_nlive, (unsigned)__popc(ml));
  }
  off = __shfl_sync(0xffffffffu, off, 0);
  if (have_out) {
    float4 *rec = s_rec + 5 * (off + __popc(mo & ((1u << lane) - 1u)));
    rec[0] = no;
    rec[1] = nd;
    rec[2] = nthr;
    rec[3] = nL;
    rec[4] = make_float4(__int_as_float(nmeta.x), __int_as_float(nmeta.y), __int_as_float(nmeta.z),
                         __int_as_float(nmeta.w));
  }
  if (wf_last_warp(&s_done)) {
    const unsigned n_out = *static_cast<volatile unsigned *>(&s_nout);
    int at = 0;
    if (lane == 0) {
      if (n_out) at = atomicAdd(&W.ctl->count[qi ^ 1], (int)n_out);
      const unsigned n_end = *static_cast<volatile unsigned *>(&s_nend);
      const unsigned n_live = *static_cast<volatile unsigned *>(&s_nlive);
      if (n_end) atomicAdd(&W.ctl->paths_done, (unsigned long long)n_end);
      if (n_live) atomicAdd(&W.ctl->segments, (unsigned long long)n_live);
    }
    at = __shfl_sync(0xffffffffu, at, 0);
    const volatile float4 *vr = s_rec;
    for (unsigned i = lane; i < n_out; i += 32) {
      const volatile float4 *rec = vr + 5 * i;
      const int slot = at + (int)i;
      out.o[slot] = make_float4(rec[0].x, rec[0].y, rec[0].z, rec[0].w);
      out.d[slot] = make_float4(rec[1].x, rec[1].y, rec[1].z, rec[1].w);
      out.thr[slot] = make_float4(rec[2].x, rec[2].y, rec[2].z, rec[2].w);
      out.L[slot] = make_float4(rec[3].x, rec[3].y, rec[3].z, rec[3].w);
      out.meta[slot] = make_int4(__float_as_int(rec[4].x), __float_as_int(rec[4].y), __float_as_int(rec[4].z),
                                 __float_as_int(rec[4].w));
    }
  }
}

// Resets the live count of the queue the next shade writes into, and the march list.
// After a shade launch into queue qo: the free slots of queue qo (from the
// survivors' count to the capacity) take the next work items, as many as
// remain (one thread).
__global__ void k_wf_regen_plan(WfCtl *ctl, int qo, int capacity) {
  const int S = ctl->count[qo];
  const unsigned long long P = ctl->next_path, T = ctl->total_paths;
  const unsigned long long room = (unsigned long long)(capacity > S ? capacity - S : 0);
  const unsigned long long n = P < T ? (T - P < room ? T - P : room) : 0ull;
  ctl->regen_item = P;
  ctl->regen_slot = S;
  ctl->regen_n = (int)n;
  ctl->next_path = P + n;
  ctl->count[qo] = S + (int)n;
}

// New camera paths into the planned slots: slot regen_slot + t takes work
// item regen_item + t (consecutive items: neighbouring pixels of one sample,
// so a warp's camera rays start together).
__global__ void k_wf_regen(const RB_GRID_CONST WfParams W, const RB_GRID_CONST WfQueue q) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= W.ctl->regen_n) return;
  wf_emit_camera(W, q, W.ctl->regen_slot + t, W.ctl->regen_item + (unsigned long long)t);
}

__global__ void k_wf_reset(WfCtl *ctl, int qi) {
  ctl->count[qi] = 0;
  ctl->march_count = 0;
  ctl->march_next = 0;
}

struct WfEngine {
  int capacity = 0;
  WfQueue q[2];
  WfCtl *ctl = nullptr;
  WfCtl *h_ctl = nullptr;
  cudaStream_t st = nullptr;
  // smooth-SDF march buffers, allocated on first use: RB_SDF_CAND x capacity
  // candidate records, counts and the march list
  int4 *cand = nullptr;
  int *ncand = nullptr;
  int *list = nullptr;
  // job table: pinned staging and device copy
  WfJob *h_jobs = nullptr;
  WfJob *d_jobs = nullptr;
  int jobs_cap = 0;
  // the last run's 8-iteration graph, reused while its launch parameters (the
  // bytes of key) are the same: a serving loop runs the engine every iteration
  struct GraphKey {
    WfParams W;
    int march_grid;
    int variant;
  } key;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t fence = nullptr;
};

// Frees everything the engine holds and nulls the pointers, so that a second
// call (after a failed allocation) frees nothing twice.
static void wf_free(WfEngine &E) {
  for (int i = 0; i < 2; ++i) {
    cudaFree(E.q[i].o); cudaFree(E.q[i].d); cudaFree(E.q[i].thr); cudaFree(E.q[i].L);
    cudaFree(E.q[i].hit); cudaFree(E.q[i].sn); cudaFree(E.q[i].meta);
  }
  std::memset(&E.q, 0, sizeof E.q);
  cudaFree(E.ctl);
  cudaFreeHost(E.h_ctl);
  E.ctl = nullptr;
  E.h_ctl = nullptr;
  cudaFree(E.cand);
  cudaFree(E.ncand);
  cudaFree(E.list);
  E.cand = nullptr;
  E.ncand = E.list = nullptr;
  cudaFreeHost(E.h_jobs);
  cudaFree(E.d_jobs);
  E.h_jobs = E.d_jobs = nullptr;
  E.jobs_cap = 0;
  if (E.graph) cudaGraphExecDestroy(E.graph);
  E.graph = nullptr;
}

static bool wf_alloc_march(WfEngine &E) {
  if (E.cand) return true;
  return cuda_ok(cudaMalloc(&E.cand, sizeof(int4) * RB_SDF_CAND * (size_t)E.capacity), "wavefront candidates") &&
         cuda_ok(cudaMalloc(&E.ncand, sizeof(int) * (size_t)E.capacity), "wavefront candidates") &&
         cuda_ok(cudaMalloc(&E.list, sizeof(int) * (size_t)E.capacity), "wavefront march list");
}

static bool wf_alloc(WfEngine &E, int capacity) {
  std::memset(&E.q, 0, sizeof E.q);
  E.capacity = capacity;
  if (injected_alloc_failure(RB_SITE_WAVEFRONT)) {
    set_error("wavefront queue: out of memory (injected)");
    return false;
  }
  bool ok = true;
  for (int i = 0; i < 2 && ok; ++i) {
    ok = cuda_ok(cudaMalloc(&E.q[i].o, sizeof(float4) * capacity), "wavefront queue") &&
         cuda_ok(cudaMalloc(&E.q[i].d, sizeof(float4) * capacity), "wavefront queue") &&
         cuda_ok(cudaMalloc(&E.q[i].thr, sizeof(float4) * capacity), "wavefront queue") &&
         cuda_ok(cudaMalloc(&E.q[i].L, sizeof(float4) * capacity), "wavefront queue") &&
         cuda_ok(cudaMalloc(&E.q[i].hit, sizeof(float4) * capacity), "wavefront queue") &&
         cuda_ok(cudaMalloc(&E.q[i].sn, sizeof(float4) * capacity), "wavefront queue") &&
         cuda_ok(cudaMalloc(&E.q[i].meta, sizeof(int4) * capacity), "wavefront queue");
  }
  ok = ok && cuda_ok(cudaMalloc(&E.ctl, sizeof(WfCtl)), "wavefront ctl") &&
       cuda_ok(cudaMallocHost(&E.h_ctl, sizeof(WfCtl)), "wavefront ctl");
  return ok;
}

// Shared-memory bytes of the staged SDF table (0 when it does not fit in 48 KB).
#ifndef WF_STAGE_SDF_TABLE
#define WF_STAGE_SDF_TABLE 1
#endif
static size_t wf_table_bytes(const WfParams &W) {
  const size_t b = sizeof(SdfPrim) * (size_t)W.S.num_sdf;
  return b <= 48 * 1024 ? b : 0;
}

// Candidate sets as bit masks when the field's table fits the mask and is
// staged in shared memory (the march reads each window's sphere from it).
static bool wf_use_mask(const WfParams &W) {
  return WF_SDF_MASK && WF_STAGE_SDF_TABLE && W.cand && W.S.num_sdf > 0 && W.S.num_sdf <= RB_SDF_MASK_BITS &&
         wf_table_bytes(W) > 0;
}

template <int MS, bool NEE>
static void wf_iteration(const WfParams &W, WfEngine &E, int qi, int grid, int march_grid, cudaStream_t st) {
  const size_t sm = stack_smem_bytes(W.S.short_stack, 256);
  const bool mask = wf_use_mask(W);
  k_wf_reset<<<1, 1, 0, st>>>(E.ctl, qi ^ 1);
  if (mask) k_wf_extend<MS, true><<<grid, 256, sm, st>>>(W, E.q[qi], qi);
  else k_wf_extend<MS, false><<<grid, 256, sm, st>>>(W, E.q[qi], qi);
  if (march_grid > 0) {
    const size_t tab = WF_STAGE_SDF_TABLE ? wf_table_bytes(W) : 0;
    if (mask) k_wf_march<MS, true><<<march_grid, 256, tab, st>>>(W, E.q[qi], 1);
    else k_wf_march<MS, false><<<march_grid, 256, tab, st>>>(W, E.q[qi], tab > 0 ? 1 : 0);
  }
  const int shade_grid = (E.capacity + WF_SHADE_THREADS - 1) / WF_SHADE_THREADS;
  // the shared stack's entries, within the 48 KB a block has beside the
  // kernel's 20 KB of staged survivors (stack_init clamps the depth to what
  // the launch provides: 8 entries by default, at most 13 here)
  const size_t shade_sm = std::min(stack_smem_bytes(W.S.short_stack, WF_SHADE_THREADS),
                                   (size_t)48 * 1024 - sizeof(float4) * 5 * WF_SHADE_THREADS - 256);
  k_wf_shade<MS, NEE><<<shade_grid, WF_SHADE_THREADS, shade_sm, st>>>(W, E.q[qi], E.q[qi ^ 1], qi);
  k_wf_regen_plan<<<1, 1, 0, st>>>(E.ctl, qi ^ 1, E.capacity);
  k_wf_regen<<<grid, 256, 0, st>>>(W, E.q[qi ^ 1]);
}

template <int MS, bool NEE>
static int wf_run(WfParams W, WfEngine &E, cudaStream_t st, int *iterations) {
  const int grid = (E.capacity + 255) / 256;
  int march_grid = 0;
  if (MS >= RB_MS_SDF && W.cand) {  // persistent march: the resident blocks
    int per_sm = 0, dev = 0, sms = 148;
    if (wf_use_mask(W))
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wf_march<MS, true>, 256, wf_table_bytes(W));
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wf_march<MS, false>, 256,
                                                    WF_STAGE_SDF_TABLE ? wf_table_bytes(W) : 0);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    march_grid = std::max(1, per_sm) * sms;
  }
  k_wf_fill<<<grid, 256, 0, st>>>(W, E.q[0], 0, E.capacity);
  g_launches++;
  // eight iterations per graph (queues 0->1->0 ...), replayed until empty;
  // the graph is kept for the next run with the same launch parameters
  WfEngine::GraphKey key;
  std::memset(&key, 0, sizeof key);
  std::memcpy(&key.W, &W, sizeof W);
  key.march_grid = march_grid;
  key.variant = MS * 2 + (NEE ? 1 : 0);
  if (!E.graph || std::memcmp(&key, &E.key, sizeof key) != 0) {
    if (E.graph) cudaGraphExecDestroy(E.graph);
    E.graph = nullptr;
    cudaGraph_t g = nullptr;
    if (!cuda_ok(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "wavefront capture"))
      return RB_ERR_CUDA;
    for (int i = 0; i < 8; ++i) wf_iteration<MS, NEE>(W, E, i & 1, grid, march_grid, st);
    const cudaError_t ec = cudaStreamEndCapture(st, &g);  // always end the capture, also after an error
    if (!cuda_ok(ec, "wavefront capture") || !g) return RB_ERR_CUDA;
    const bool inst = cuda_ok(cudaGraphInstantiate(&E.graph, g, 0), "wavefront graph");
    cudaGraphDestroy(g);
    if (!inst) {
      E.graph = nullptr;
      return RB_ERR_CUDA;
    }
    std::memcpy(&E.key, &key, sizeof key);
  }
  int it = 0;
  for (int guard = 0; guard < 1 << 20; ++guard) {
    cudaGraphLaunch(E.graph, st);
    g_launches += march_grid > 0 ? 48 : 40;
    it += 8;
    cudaMemcpyAsync(E.h_ctl, E.ctl, sizeof(WfCtl), cudaMemcpyDeviceToHost, st);
    if (!cuda_ok(cudaStreamSynchronize(st), "wavefront iteration")) {
      cudaGraphExecDestroy(E.graph);
      E.graph = nullptr;
      return RB_ERR_CUDA;
    }
    if (E.h_ctl->count[0] == 0) break;  // eight iterations end in queue 0
  }
  if (iterations) *iterations = it;
  return RB_OK;
}


// Runs the engine over `njobs` jobs of one scene (host job table; item_begin
// filled here) until every path has ended. The engine records its iterations
// into a CUDA graph, which needs a capturable stream: it runs on a private
// non-blocking stream ordered after the caller's stream on entry and before
// it on return. Queues, march buffers and the job table are kept per
// (thread, device) between calls. counters (host, may be null): segments,
// paths, stack overflows, iterations.
int wf_render_jobs(const DeviceScene *ds, WfJob *jobs, int njobs, int queue_capacity, uint64_t *counters,
                   cudaStream_t caller) {
  static thread_local cudaStream_t priv[64] = {nullptr};
  static thread_local WfEngine cached[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return RB_ERR_UNSUPPORTED;
  if (!priv[dev] && !cuda_ok(cudaStreamCreateWithFlags(&priv[dev], cudaStreamNonBlocking), "wavefront stream"))
    return RB_ERR_CUDA;
  cudaStream_t st = priv[dev];
  const int cap = queue_capacity > 0 ? queue_capacity : ds->wf_queue > 0 ? ds->wf_queue : (1 << 20);
  WfEngine &E = cached[dev];
  if (E.capacity != cap) {
    if (E.capacity) wf_free(E);
    E.capacity = 0;
    if (!wf_alloc(E, cap)) {
      wf_free(E);
      E.capacity = 0;
      return RB_ERR_OUT_OF_MEMORY;
    }
  }
  // the previous run synchronised its stream, so the staging table is free
  if (njobs > E.jobs_cap) {
    cudaFreeHost(E.h_jobs);
    cudaFree(E.d_jobs);
    E.h_jobs = E.d_jobs = nullptr;
    E.jobs_cap = 0;
    if (!cuda_ok(cudaMallocHost(&E.h_jobs, sizeof(WfJob) * njobs), "wavefront job table") ||
        !cuda_ok(cudaMalloc(&E.d_jobs, sizeof(WfJob) * njobs), "wavefront job table"))
      return RB_ERR_OUT_OF_MEMORY;
    E.jobs_cap = njobs;
  }
  unsigned long long total = 0;
  bool nee = false;
  for (int j = 0; j < njobs; ++j) {
    jobs[j].item_begin = total;
    total += (unsigned long long)jobs[j].P.width * jobs[j].P.height * (unsigned long long)jobs[j].P.samples;
    nee = nee || jobs[j].G.nee != 0;
  }
  const bool field = ds->ms >= RB_MS_SDF && ds->view.sdf_k > 0.0f && ds->view.num_sdf > 0;
  if (field && !wf_alloc_march(E)) return RB_ERR_OUT_OF_MEMORY;
  if (total == 0) return RB_OK;  // (a call without work only allocates)
  std::memcpy(E.h_jobs, jobs, sizeof(WfJob) * njobs);
  WfParams W;
  std::memset(&W, 0, sizeof W);
  W.S = ds->view;
  W.jobs = E.d_jobs;
  W.njobs = njobs;
  W.ctl = E.ctl;
  if (field) {
    W.cand = E.cand;
    W.ncand = E.ncand;
    W.list = E.list;
    W.cap = E.capacity;
  }
  if (!E.fence && !cuda_ok(cudaEventCreateWithFlags(&E.fence, cudaEventDisableTiming), "wavefront fence"))
    return RB_ERR_CUDA;
  cudaEvent_t fence = E.fence;
  cudaEventRecord(fence, caller);
  cudaStreamWaitEvent(st, fence, 0);
  cudaMemcpyAsync(E.d_jobs, E.h_jobs, sizeof(WfJob) * njobs, cudaMemcpyHostToDevice, st);
  WfCtl init;
  std::memset(&init, 0, sizeof init);
  init.total_paths = total;
  cudaMemcpyAsync(E.ctl, &init, sizeof init, cudaMemcpyHostToDevice, st);
  int it = 0, rc;
  switch (ds->ms) {
    case RB_MS_DIFFUSE: rc = nee ? wf_run<RB_MS_DIFFUSE, true>(W, E, st, &it) : wf_run<RB_MS_DIFFUSE, false>(W, E, st, &it); break;
    case RB_MS_CLASSIC: rc = nee ? wf_run<RB_MS_CLASSIC, true>(W, E, st, &it) : wf_run<RB_MS_CLASSIC, false>(W, E, st, &it); break;
    case RB_MS_FULL: rc = nee ? wf_run<RB_MS_FULL, true>(W, E, st, &it) : wf_run<RB_MS_FULL, false>(W, E, st, &it); break;
    default: rc = nee ? wf_run<RB_MS_SDF, true>(W, E, st, &it) : wf_run<RB_MS_SDF, false>(W, E, st, &it); break;
  }
  if (rc == RB_OK && counters) {
    counters[0] = E.h_ctl->segments;
    counters[1] = E.h_ctl->paths_done;
    counters[2] = E.h_ctl->overflow;
    counters[3] = (uint64_t)it;
  }
  cudaEventRecord(fence, st);
  cudaStreamWaitEvent(caller, fence, 0);
  cudaStreamSynchronize(st);
  return rc;
}

static WfJob wf_job(const double *frame, int width, int height, int samples, int sample_base, int max_depth,
                    uint32_t salt, double *acc) {
  WfJob J;
  std::memset(&J, 0, sizeof J);
  J.P = frame_from(frame, width, height);
  J.P.samples = samples;
  J.P.sample_base = sample_base;
  J.P.max_depth = max_depth;
  J.P.seed = current_opts().seed;
  J.P.salt = salt;
  J.G = current_globals();
  J.acc = acc;
  return J;
}

}  // namespace rb

using namespace rb;

extern "C" int rb_render_wavefront(const rb_cuda_scene *scene, int width, int height, const double frame[21],
                                   int samples, int sample_base, int max_depth, double *accum, int queue_capacity,
                                   uint64_t *counters, void *stream) {
  DeviceScene *ds = lookup_scene(scene);
  if (!ds) {
    set_error("rb_render_wavefront: unknown scene handle");
    return RB_ERR_NOT_FOUND;
  }
  if (width <= 0 || height <= 0 || !frame || !accum || samples < 0 || max_depth < 0 || sample_base < 0) {
    set_error("rb_render_wavefront: invalid argument");
    return RB_ERR_INVALID_ARG;
  }
  if (samples == 0 || max_depth == 0) return RB_OK;
  WfJob J = wf_job(frame, width, height, samples, sample_base, max_depth, 0u, accum);
  uint64_t c[4] = {0, 0, 0, 0};
  cudaStream_t caller = static_cast<cudaStream_t>(stream);
  const int rc = wf_render_jobs(ds, &J, 1, queue_capacity, c, caller);
  if (rc == RB_OK && counters) cudaMemcpyAsync(counters, c, sizeof c, cudaMemcpyHostToDevice, caller);
  return rc;
}

extern "C" int rb_render_views_wavefront(const rb_cuda_scene *scene, int n_views, int width, int height,
                                         const double *frames, int samples, int sample_base, int max_depth,
                                         double *accum, int queue_capacity, uint64_t *counters, void *stream) {
  DeviceScene *ds = lookup_scene(scene);
  if (!ds) {
    set_error("rb_render_views_wavefront: unknown scene handle");
    return RB_ERR_NOT_FOUND;
  }
  if (n_views <= 0 || n_views > 4096 || width <= 0 || height <= 0 || !frames || !accum || samples < 0 ||
      max_depth < 0 || sample_base < 0) {
    set_error("rb_render_views_wavefront: invalid argument");
    return RB_ERR_INVALID_ARG;
  }
  if (samples == 0 || max_depth == 0) return RB_OK;
  std::vector<WfJob> jobs((size_t)n_views);
  const size_t npx = (size_t)width * height;
  for (int v = 0; v < n_views; ++v)
    jobs[v] = wf_job(frames + 21 * (size_t)v, width, height, samples, sample_base, max_depth, (uint32_t)v,
                     accum + 4 * npx * v);
  uint64_t c[4] = {0, 0, 0, 0};
  cudaStream_t caller = static_cast<cudaStream_t>(stream);
  const int rc = wf_render_jobs(ds, jobs.data(), n_views, queue_capacity, c, caller);
  if (rc == RB_OK && counters) cudaMemcpyAsync(counters, c, sizeof c, cudaMemcpyHostToDevice, caller);
  return rc;
}
