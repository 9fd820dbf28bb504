// Batched multi-job engine and the serving loop.
//
// One persistent launch per iteration renders every active job: the
// iteration's work is a list of pixel tasks (job, pixel, n samples) that warps
// claim 32 at a time with one atomic per warp (ballot of the lanes that need
// work). A lane traces its task's samples one whole path at a time (the
// warp's camera rays start together, as in the per-frame kernel) and claims
// the next task the moment its pixel is done, so lanes stay busy across task
// and job boundaries and one launch fills the GPU whatever the jobs' sizes.
// A task owns its pixel for the launch, so the pixel's sums are updated
// without atomics (Kahan in FP32, or FP64).
//
// The serving loop (rb_server_*) keeps scenes resident, admits queued jobs as
// slots and the HBM budget allow (continuous batching: new jobs join the next
// iteration while others are still running), gives every active job a share
// of the iteration's path quantum, retires finished jobs and optionally writes
// a u8 progressive frame per job. Each iteration (job-table upload, counter
// reset, kernel) can be one CUDA graph launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "rb_path.cuh"

namespace rb {

extern std::atomic<unsigned long long> g_launches;
DeviceScene *lookup_scene(const void *handle);

struct __align__(16) BatchJob {
  SceneView S;
  FrameF P;          // P.samples = samples per pixel in this iteration
  Globals G;
  float4 *acc;       // FP32 sums (w*h) followed by Kahan compensation (w*h)
  double *acc64;     // FP64 sums (w*h*4), or null
  unsigned char *frame;  // u8 RGBA progressive frame or null
  long long task_begin;  // first task of this job in the iteration
  int spp_total;         // samples accumulated after this iteration (frame normalisation)
  int pad[3];
};

// Control blocks: [0] all jobs (frames), [1..8] one per launch group
// (kernel class 1-4, plus 4 for the next-event-estimation variant).
#define RB_GROUPS 9

struct BatchCtl {
  unsigned long long next_task;
  unsigned long long total_tasks;
  unsigned long long segments;
  unsigned long long paths;
  unsigned long long overflow;
  int njobs;
  int job_offset;  // first job of this launch's class in the job table
  int pad[4];
};

// The scene and settings shared by every job of one batched launch.
struct BatchUniform {
  SceneView S;
  Globals G;
};

__device__ __forceinline__ int find_job(const BatchJob *__restrict__ jobs, int njobs, long long t) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&jobs[mid].task_begin) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Scene and settings of a lane's job: the launch's own (kernel parameters,
// read through the constant bank) when every job of the launch shares them
// (UNI), else the job table's record (global loads every path segment).
template <bool UNI, class T>
__device__ __forceinline__ const T &job_or_uniform(const T &uniform, const T &job) {
  if constexpr (UNI) return uniform;
  else return job;
}

template <int MS, int MINB, bool NEE, bool UNI>
__global__ void __launch_bounds__(256, MINB) k_batch(const BatchJob *__restrict__ jobs, BatchCtl *__restrict__ ctl,
                                                     const SceneView Su, const Globals Gu) {
  extern __shared__ int2 smem[];
  jobs += ctl->job_offset;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  // shared stack entries: as many as the launch provided (the largest of its
  // jobs' scenes' short_stack)
  Stack st;
  stack_init(st, smem, tid, blockDim.x, RB_SHORT_MAX);
  uint32_t ovf = 0;
  const unsigned long long total = ctl->total_tasks;
  const int njobs = ctl->njobs;
  unsigned long long segs = 0, paths = 0;

  bool have = false, done_all = false;
  int j = 0, pix = 0, x = 0, y = 0, s = 0, nsamp = 0, bounce = 0;
  bool alive = false;
  Ray ray;
  f3 thr(1.f, 1.f, 1.f), L(0.f, 0.f, 0.f);
  float sx = 0.f, sy = 0.f, sz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f, prev_pdf = 0.f;
  uint32_t key = 0;
  while (true) {
    // claim tasks for idle lanes, one atomic per warp
    const bool need = !have && !done_all;
    const unsigned mask = __ballot_sync(0xffffffffu, need);
    if (mask) {
      unsigned long long base = 0;
      const int leader = __ffs(mask) - 1;
      if (lane == leader) base = atomicAdd(&ctl->next_task, (unsigned long long)__popc(mask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const unsigned long long t = base + __popc(mask & ((1u << lane) - 1u));
        if (t < total) {
          j = find_job(jobs, njobs, (long long)t);
          pix = (int)((long long)t - __ldg(&jobs[j].task_begin));
          const int w = __ldg(&jobs[j].P.width);
          x = pix % w;
          y = pix / w;
          nsamp = __ldg(&jobs[j].P.samples);
          s = 0;
          sx = sy = sz = cx = cy = cz = 0.f;
          have = true;
          alive = false;
        } else {
          done_all = true;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, have) == 0) break;  // every lane out of work
    if (have) {
      const BatchJob &J = jobs[j];
      if (!alive) {
        if (s < nsamp && J.P.max_depth > 0) {
          key = rb_path_key(J.P.seed, J.P.salt, (uint32_t)pix, (uint32_t)(J.P.sample_base + s));
          ++s;
          ray = camera_ray(J.P, job_or_uniform<UNI>(Gu, J.G), x, y, key);
          thr = f3(1.f, 1.f, 1.f);
          L = f3(0.f, 0.f, 0.f);
          bounce = 0;
          prev_pdf = 0.f;
          alive = true;
        } else {
          // task complete: fold the samples into the pixel (this task owns it)
          const int n = J.P.width * J.P.height;
          if (J.acc64) {
            double4 *a = reinterpret_cast<double4 *>(J.acc64) + pix;
            double4 v = *a;
            v.x += (double)sx - (double)cx;
            v.y += (double)sy - (double)cy;
            v.z += (double)sz - (double)cz;
            *a = v;
          } else {
            float4 a = J.acc[pix], c = J.acc[n + pix];
            kahan_add(a.x, c.x, sx - cx);
            kahan_add(a.y, c.y, sy - cy);
            kahan_add(a.z, c.z, sz - cz);
            J.acc[pix] = a;
            J.acc[n + pix] = c;
          }
          paths += (unsigned long long)nsamp;
          have = false;
        }
      }
      if (alive) {
        // Diffuse scenes (Lambert walls, long paths of geometrically
        // distributed length): one segment per pass of the outer loop, so a
        // lane whose path ends starts its next sample (or claims its next
        // task) at once, as the per-frame kernel's flattened loop does. The
        // other classes trace the whole path at once: a lane whose path ends
        // early waits for the warp's longest, and the warp's next camera rays
        // start together (coherent).
        constexpr bool kFlat = MS == RB_MS_DIFFUSE;
        bool end = false;
        do {
          ++segs;
          end = path_segment<NEE, MS>(job_or_uniform<UNI>(Su, J.S), job_or_uniform<UNI>(Gu, J.G), st, ovf, ray, thr, L,
                                      bounce, prev_pdf, key, J.P.max_depth);
        } while (!kFlat && !end);
        if (end) {
          kahan_add(sx, cx, L.x);
          kahan_add(sy, cy, L.y);
          kahan_add(sz, cz, L.z);
          alive = false;
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    segs += __shfl_down_sync(0xffffffffu, segs, o);
    paths += __shfl_down_sync(0xffffffffu, paths, o);
  }
  if (lane == 0) {
    atomicAdd(&ctl->segments, segs);
    atomicAdd(&ctl->paths, paths);
  }
  if (ovf) atomicAdd(&ctl->overflow, (unsigned long long)ovf);
}

// u8 RGBA progressive frames of all jobs of the iteration (one thread per pixel of every job).
__global__ void k_batch_frames(const BatchJob *__restrict__ jobs, const BatchCtl *__restrict__ ctl) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ctl->total_tasks) return;
  const int j = find_job(jobs, ctl->njobs, t);
  const BatchJob &J = jobs[j];
  if (!J.frame) return;
  const int pix = (int)(t - J.task_begin);
  const int n = J.P.width * J.P.height;
  float r, g, b;
  if (J.acc64) {
    const double4 v = reinterpret_cast<const double4 *>(J.acc64)[pix];
    r = (float)v.x; g = (float)v.y; b = (float)v.z;
  } else {
    const float4 a = J.acc[pix], c = J.acc[n + pix];
    r = a.x - c.x; g = a.y - c.y; b = a.z - c.z;
  }
  const float inv = 1.0f / (float)max(J.spp_total, 1);
  unsigned char *o = J.frame + 4 * (size_t)pix;
  o[0] = (unsigned char)(256.0f * fminf(sqrtf(fmaxf(r * inv, 0.0f)), 0.999f));
  o[1] = (unsigned char)(256.0f * fminf(sqrtf(fmaxf(g * inv, 0.0f)), 0.999f));
  o[2] = (unsigned char)(256.0f * fminf(sqrtf(fmaxf(b * inv, 0.0f)), 0.999f));
  o[3] = 255;
}

template <int MS, bool NEE>
// uni (may be null): the scene and settings every job of the launch shares;
// the uniform variant exists for the default occupancy (4 blocks per SM).
static void launch_batch_ms(int minb, int grid, cudaStream_t st, const BatchJob *jobs, BatchCtl *ctl,
                            const BatchUniform *uni, int short_stack) {
  const size_t sm = stack_smem_bytes(short_stack, 256);
  if (uni && minb == 4) {
    k_batch<MS, 4, NEE, true><<<grid, 256, sm, st>>>(jobs, ctl, uni->S, uni->G);
    return;
  }
  SceneView s0;
  Globals g0;
  std::memset(&s0, 0, sizeof s0);
  std::memset(&g0, 0, sizeof g0);
  switch (minb) {
    case 1: k_batch<MS, 1, NEE, false><<<grid, 256, sm, st>>>(jobs, ctl, s0, g0); break;
    case 3: k_batch<MS, 3, NEE, false><<<grid, 256, sm, st>>>(jobs, ctl, s0, g0); break;
    case 4: k_batch<MS, 4, NEE, false><<<grid, 256, sm, st>>>(jobs, ctl, s0, g0); break;
    default: k_batch<MS, 2, NEE, false><<<grid, 256, sm, st>>>(jobs, ctl, s0, g0); break;
  }
}

// Resident 256-thread blocks per SM of the batched kernel (its register
// budget): 4 for every class, from a sweep on B200 (icosphere, One-Weekend,
// SDF-field and Cornell views); overridden by rb_server_opts.occupancy /
// rb_render_opts.reserved[0].
static int batch_minb(int ms, bool nee) {
  (void)ms;
  (void)nee;
  return 4;
}

// One persistent launch for a class group; the next-event-estimation variant
// only when a job of the group asks for it (it costs registers).
// short_stack: the largest SceneView::short_stack among the launch's jobs.
static void launch_batch(int ms, int minb, bool nee, cudaStream_t st, const BatchJob *jobs, BatchCtl *ctl, int sms,
                         const BatchUniform *uni, int short_stack) {
  const int grid = sms * minb;  // persistent: exactly the resident blocks
  if (nee) {
    if (ms == RB_MS_DIFFUSE) launch_batch_ms<RB_MS_DIFFUSE, true>(minb, grid, st, jobs, ctl, uni, short_stack);
    else if (ms == RB_MS_CLASSIC) launch_batch_ms<RB_MS_CLASSIC, true>(minb, grid, st, jobs, ctl, uni, short_stack);
    else if (ms == RB_MS_FULL) launch_batch_ms<RB_MS_FULL, true>(minb, grid, st, jobs, ctl, uni, short_stack);
    else launch_batch_ms<RB_MS_SDF, true>(minb, grid, st, jobs, ctl, uni, short_stack);
  } else {
    if (ms == RB_MS_DIFFUSE) launch_batch_ms<RB_MS_DIFFUSE, false>(minb, grid, st, jobs, ctl, uni, short_stack);
    else if (ms == RB_MS_CLASSIC) launch_batch_ms<RB_MS_CLASSIC, false>(minb, grid, st, jobs, ctl, uni, short_stack);
    else if (ms == RB_MS_FULL) launch_batch_ms<RB_MS_FULL, false>(minb, grid, st, jobs, ctl, uni, short_stack);
    else launch_batch_ms<RB_MS_SDF, false>(minb, grid, st, jobs, ctl, uni, short_stack);
  }
  g_launches++;
}

// Loads every batched-kernel variant up front so that lazy module loading
// does not land inside a timed iteration.
template <int MS>
static void preload_ms() {
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, k_batch<MS, 1, false, false>);
  cudaFuncGetAttributes(&a, k_batch<MS, 2, false, false>);
  cudaFuncGetAttributes(&a, k_batch<MS, 3, false, false>);
  cudaFuncGetAttributes(&a, k_batch<MS, 4, false, false>);
  cudaFuncGetAttributes(&a, k_batch<MS, 4, false, true>);
  cudaFuncGetAttributes(&a, k_batch<MS, 1, true, false>);
  cudaFuncGetAttributes(&a, k_batch<MS, 2, true, false>);
  cudaFuncGetAttributes(&a, k_batch<MS, 3, true, false>);
  cudaFuncGetAttributes(&a, k_batch<MS, 4, true, false>);
  cudaFuncGetAttributes(&a, k_batch<MS, 4, true, true>);
}
static void preload_batch_kernels() {
  preload_ms<RB_MS_DIFFUSE>();
  preload_ms<RB_MS_CLASSIC>();
  preload_ms<RB_MS_FULL>();
  preload_ms<RB_MS_SDF>();
  cudaFuncAttributes a;
  cudaFuncGetAttributes(&a, k_batch_frames);
}

// ---------------------------------------------------------------------------
// Serving loop
// ---------------------------------------------------------------------------
struct Job {
  rb_job_request req;
  int64_t id;
  int state = 0;  // 0 queued, 1 active, 2 done, -1 rejected
  int spp_done = 0;
  double t_arrival = 0, t_admit = 0, t_done = 0;
  float4 *acc = nullptr;
  double *acc64 = nullptr;
  unsigned char *frame = nullptr;
  float *lum = nullptr;       // mean luminance at the last convergence check (converging jobs)
  bool converged = false;
  int64_t bytes = 0;
  int error = 0;  // rb_status of a rejection
};

#define RB_PF_STREAMS 4

struct Server {
  rb_server_opts o;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  int sms = 148;
  std::vector<const DeviceScene *> scenes;
  std::unordered_map<int64_t, Job> jobs;
  std::deque<int64_t> queue;
  std::vector<int64_t> active;
  int64_t next_id = 0;
  int64_t used_bytes = 0, peak_bytes = 0;
  // path slots of the wavefront engine: one capacity for all of the server's
  // smooth-SDF scenes (the largest tuned one), so that runs never reallocate
  int wf_cap = 0;
  BatchJob *h_jobs = nullptr;  // pinned
  BatchJob *d_jobs = nullptr;
  BatchCtl *h_ctl = nullptr;   // pinned
  BatchCtl *d_ctl = nullptr;
  unsigned long long *h_conv = nullptr, *d_conv = nullptr;  // converged-pixel counts per planned job
  unsigned long long *h_pfc = nullptr, *d_pfc = nullptr;    // per-frame launches' counters of an iteration
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // wavefront jobs run on their own stream beside the class kernels: ev_up
  // marks the iteration's uploads, ev_wf the end of its wavefront runs
  cudaStream_t st_wf = nullptr;
  cudaEvent_t ev_up = nullptr, ev_wf = nullptr;
  // per-frame jobs of an iteration run round-robin on RB_PF_STREAMS streams
  // forked after the uploads (ev_pf_fork) and joined before the iteration's
  // counters are read, so one job's launch tail overlaps the next job's work
  // and the class kernels
  cudaStream_t st_pf[RB_PF_STREAMS] = {};
  cudaEvent_t ev_pf_fork = nullptr, ev_pf_join[RB_PF_STREAMS] = {};
  // job buffers come from a private stream-ordered pool that keeps freed
  // memory (the device's default pool hands it back at every synchronisation,
  // and mapping it again on the next admission stalls the loop)
  cudaMemPool_t pool = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_frames = -1;
  // per class group: the scene shared by all its jobs (-1: none or several)
  // and their shared settings, as the graph's kernels were captured with
  int graph_scene[RB_GROUPS];
  Globals graph_G[RB_GROUPS];
  double aging = 0.5;  // priority = remaining paths / (1 + aging * seconds waited)
  std::chrono::steady_clock::time_point t0;
  rb_server_stats stats;
  std::vector<double> latencies;
  double first_arrival = -1, last_done = 0;
  int64_t quantum = 0;        // path quantum of the next iteration
  double last_ms = 0.0;       // device time of the last iteration

  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

static int64_t job_bytes(const rb_job_request &r, bool frames) {
  const int64_t n = (int64_t)r.width * r.height;
  return n * 32 + (frames ? n * 4 : 0) + (r.converge_threshold > 0.0f ? n * 4 : 0);
}

// Per-job convergence count: the per-pixel luminance test of the reference's
// adaptive sampling (render_acc_kernel.cu:241-271) between the job's last
// check (lum) and its sums now (spp_now samples). As in the reference a
// converged pixel stays converged: lum holds -1 - (its luminance) from then
// on (the reference keeps the flag in the sign of its sample count). Counts
// the converged pixels.
__global__ void k_job_converge(const float4 *__restrict__ acc, const double *__restrict__ acc64, float *lum, int n,
                               int spp_now, int checked_before, float threshold, unsigned long long *count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool conv = false;
  if (i < n) {
    float r, g, b;
    if (acc64) {
      const double4 v = reinterpret_cast<const double4 *>(acc64)[i];
      r = (float)v.x; g = (float)v.y; b = (float)v.z;
    } else {
      const float4 a = acc[i], c = acc[n + i];
      r = a.x - c.x; g = a.y - c.y; b = a.z - c.z;
    }
    const float lum_before = lum[i];
    if (lum_before < 0.0f) {
      conv = true;
    } else {
      const float inv_s = 1.0f / (float)spp_now;
      const float lum_after = 0.299f * r * inv_s + 0.587f * g * inv_s + 0.114f * b * inv_s;
      conv = checked_before && fabsf(lum_after - lum_before) / fmaxf(lum_after, 0.001f) < threshold;
      lum[i] = conv ? -1.0f - lum_after : lum_after;
    }
  }
  const unsigned m = __ballot_sync(0xffffffffu, conv);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(count, (unsigned long long)__popc(m));
}

// Jobs of scenes with a smooth SDF field run on the wavefront engine, whose
// field march keeps a warp's lanes stepping together (see rb_wavefront.cu).
#define RB_WF_GROUP RB_GROUPS
// Path slots of the server's wavefront engine (8 M: about 5 GB of queues and
// SDF march buffers, held for the process beside the jobs' HBM budget);
// 4 M -> 8 M measured +4.6 % on the SDF field.
#define RB_SERVER_WF_QUEUE (1 << 23)
// the scene's autotuned path slots when it has them
static int scene_wf_queue(const DeviceScene *ds) { return ds->wf_queue > 0 ? ds->wf_queue : RB_SERVER_WF_QUEUE; }
static bool on_wavefront_scene(const Server &S, const DeviceScene *ds) {
  return S.o.wavefront_field && ds->ms >= RB_MS_SDF && ds->view.sdf_k > 0.0f && ds->view.num_sdf > 0;
}

static bool on_wavefront(const Server &S, const Job &J) { return on_wavefront_scene(S, S.scenes[J.req.scene]); }

// 1: admitted; 0: no room now (slots or budget); -1: the job's buffers could
// not be allocated (the device is out of memory).
static int admit(Server &S, Job &J) {
  const bool frames = S.o.frames_every > 0;
  const int64_t need = job_bytes(J.req, frames);
  if (S.used_bytes + need > S.o.memory_budget_bytes || (int)S.active.size() >= S.o.max_active_jobs) return 0;
  const int64_t n = (int64_t)J.req.width * J.req.height;
  const bool f64 = J.req.fp64_accum || J.req.spp > 65536 || on_wavefront(S, J);
  cudaError_t e;
  if (injected_alloc_failure(RB_SITE_SERVER_JOB)) {
    e = cudaErrorMemoryAllocation;
  } else if (f64) {
    e = cudaMallocFromPoolAsync((void **)&J.acc64, n * 32, S.pool, S.st);
    if (e == cudaSuccess) e = cudaMemsetAsync(J.acc64, 0, n * 32, S.st);
  } else {
    e = cudaMallocFromPoolAsync((void **)&J.acc, n * 32, S.pool, S.st);
    if (e == cudaSuccess) e = cudaMemsetAsync(J.acc, 0, n * 32, S.st);
  }
  if (e == cudaSuccess && frames) {
    e = cudaMallocFromPoolAsync((void **)&J.frame, n * 4, S.pool, S.st);
    if (e == cudaSuccess) e = cudaMemsetAsync(J.frame, 0, n * 4, S.st);
  }
  if (e == cudaSuccess && J.req.converge_threshold > 0.0f) {
    e = cudaMallocFromPoolAsync((void **)&J.lum, n * 4, S.pool, S.st);
    if (e == cudaSuccess) e = cudaMemsetAsync(J.lum, 0, n * 4, S.st);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (J.acc) cudaFreeAsync(J.acc, S.st);
    if (J.acc64) cudaFreeAsync(J.acc64, S.st);
    if (J.frame) cudaFreeAsync(J.frame, S.st);
    if (J.lum) cudaFreeAsync(J.lum, S.st);
    J.acc = nullptr; J.acc64 = nullptr; J.frame = nullptr; J.lum = nullptr;
    set_error(std::string("server: job ") + std::to_string(J.id) + " buffers: " + cudaGetErrorString(e));
    return -1;
  }
  J.bytes = need;
  S.used_bytes += need;
  S.peak_bytes = std::max(S.peak_bytes, S.used_bytes);
  J.state = 1;
  J.t_admit = S.now();
  S.active.push_back(J.id);
  return 1;
}

static void free_job(Server &S, Job &J) {
  if (J.acc) cudaFreeAsync(J.acc, S.st);
  if (J.acc64) cudaFreeAsync(J.acc64, S.st);
  if (J.frame) cudaFreeAsync(J.frame, S.st);
  if (J.lum) cudaFreeAsync(J.lum, S.st);
  J.acc = nullptr; J.acc64 = nullptr; J.frame = nullptr; J.lum = nullptr;
  S.used_bytes -= J.bytes;
  J.bytes = 0;
}

static int server_step(Server &S) {
  // admission: FIFO while slots and memory allow
  while (!S.queue.empty()) {
    Job &J = S.jobs[S.queue.front()];
    const int a = admit(S, J);
    if (a < 0) {  // out of device memory: reject this job, keep serving the others
      J.state = -1;
      J.error = RB_ERR_OUT_OF_MEMORY;
      S.stats.jobs_rejected++;
      S.queue.pop_front();
      continue;
    }
    if (a == 0) {
      if (S.active.empty()) {  // can never fit: reject instead of blocking the queue
        J.state = -1;
        J.error = RB_ERR_CAPACITY;
        S.stats.jobs_rejected++;
        S.queue.pop_front();
        continue;
      }
      break;
    }
    S.queue.pop_front();
  }
  if (S.active.empty()) return (int)S.queue.size();
  // Plan: shortest remaining work first, aged by waiting time so large jobs
  // are not starved, until the iteration's path quantum is used; each planned
  // job gets as many samples per pixel as fit (capped), so tasks are long and
  // an iteration holds few scenes.
  const double tnow = S.now();
  // pf: the job runs on the per-frame kernel (rb_server_opts.per_frame_classes)
  struct Plan { int64_t id; int spp; int cls; double prio; int pf; };
  std::vector<Plan> cand;
  for (int64_t id : S.active) {
    Job &J = S.jobs[id];
    const double rem = (double)J.req.width * J.req.height * (J.req.spp - J.spp_done);
    const double age = tnow - J.t_arrival;
    // group key: kernel class, plus 4 when the job uses next-event estimation
    const int cls = on_wavefront(S, J) ? RB_WF_GROUP : S.scenes[J.req.scene]->ms + (J.req.nee ? 4 : 0);
    const int ms_cls = cls > 4 ? cls - 4 : cls;
    const int pf = cls != RB_WF_GROUP && ((S.o.per_frame_classes >> ms_cls) & 1) && J.acc && !J.acc64 ? 1 : 0;
    cand.push_back({id, 0, cls, rem / (1.0 + S.aging * age), pf});
  }
  std::stable_sort(cand.begin(), cand.end(), [](const Plan &a, const Plan &b) { return a.prio < b.prio; });
  int64_t budget = S.quantum > 0 ? S.quantum : S.o.paths_per_iteration;
  std::vector<Plan> plan;
  for (Plan &c : cand) {
    if (budget <= 0 && !plan.empty()) break;
    Job &J = S.jobs[c.id];
    const int64_t px = (int64_t)J.req.width * J.req.height;
    int64_t q = std::max<int64_t>(1, budget / std::max<int64_t>(px, 1));
    // the cap bounds the batched kernel's task length; a per-frame job takes
    // what the quantum allows in one launch (each launch pays its ramp and
    // tail: on Cornell 512x512 five 51-spp launches took 16.5 ms against
    // 14.7 ms for one of 256 spp)
    if (!c.pf) q = std::min<int64_t>(q, S.o.max_spp_per_iteration);
    q = std::min<int64_t>(q, J.req.spp - J.spp_done);
    c.spp = (int)q;
    budget -= q * px;
    plan.push_back(c);
  }
  // group by kernel class (each class runs its own specialised persistent
  // kernel, so a job's code and results do not depend on the mix); within a
  // class, more samples per task first
  // per-frame jobs last, so every batched class's tasks stay contiguous
  std::stable_sort(plan.begin(), plan.end(), [](const Plan &a, const Plan &b) {
    return a.pf != b.pf ? a.pf < b.pf : a.cls != b.cls ? a.cls < b.cls : a.spp > b.spp;
  });
  long long tb = 0;
  std::memset(S.h_ctl, 0, sizeof(BatchCtl) * RB_GROUPS);
  int jfirst[RB_GROUPS] = {0};
  std::vector<size_t> wf_k;  // planned jobs that run on the wavefront engine (sorted last)
  std::vector<size_t> pf_k;  // planned jobs that run on the per-frame kernel
  for (size_t k = 0; k < plan.size(); ++k) {
    Job &J = S.jobs[plan[k].id];
    const DeviceScene *ds = S.scenes[J.req.scene];
    const int cls = plan[k].cls;
    if (cls == RB_WF_GROUP) {
      wf_k.push_back(k);
    } else if (plan[k].pf) {
      pf_k.push_back(k);
    } else {
      BatchCtl &C = S.h_ctl[cls];
      if (C.njobs == 0) {
        jfirst[cls] = (int)k;
        C.next_task = (unsigned long long)tb;
      }
      C.njobs++;
    }
    BatchJob &B = S.h_jobs[k];
    std::memset(&B, 0, sizeof B);
    B.S = ds->view;
    B.P = frame_from(J.req.frame, J.req.width, J.req.height);
    B.P.samples = plan[k].spp;
    B.P.sample_base = J.spp_done;
    B.P.max_depth = J.req.max_depth;
    B.P.seed = current_opts().seed;
    B.P.salt = J.req.seed;
    B.G.light_intensity = J.req.light_intensity;
    B.G.background_intensity = J.req.background_intensity;
    B.G.metal_fuzziness = J.req.metal_fuzziness;
    B.G.glass_ior = J.req.glass_ior;
    B.G.dof_enabled = J.req.dof_enabled;
    B.G.dof_aperture = J.req.dof_aperture;
    B.G.dof_focus = J.req.dof_focus;
    B.G.nee = J.req.nee;
    B.acc = J.acc;
    B.acc64 = J.acc64;
    B.task_begin = tb;
    B.spp_total = J.spp_done + plan[k].spp;
    const bool frame_now = S.o.frames_every > 0 && ((S.stats.iterations + 1) % S.o.frames_every == 0 ||
                                                     B.spp_total >= J.req.spp);
    B.frame = frame_now ? J.frame : nullptr;
    tb += (long long)J.req.width * J.req.height;
    if (cls != RB_WF_GROUP && !plan[k].pf) S.h_ctl[cls].total_tasks = (unsigned long long)tb;
  }
  for (int c = 1; c < RB_GROUPS; ++c) S.h_ctl[c].job_offset = jfirst[c];
  // groups whose jobs share one scene and one setting run the uniform kernel
  // (scene and settings as launch parameters); an empty group keeps what the
  // graph has, so its capture stays valid
  int uni_scene[RB_GROUPS];
  Globals uni_G[RB_GROUPS];
  for (int c = 0; c < RB_GROUPS; ++c) {
    uni_scene[c] = S.graph_scene[c];
    uni_G[c] = S.graph_G[c];
  }
  {
    bool seen[RB_GROUPS] = {false};
    for (size_t k = 0; k < plan.size(); ++k) {
      const int cls = plan[k].cls;
      if (cls == RB_WF_GROUP) continue;
      const int sc = S.jobs[plan[k].id].req.scene;
      if (!seen[cls]) {
        seen[cls] = true;
        uni_scene[cls] = sc;
        uni_G[cls] = S.h_jobs[k].G;
      } else if (uni_scene[cls] != sc || std::memcmp(&uni_G[cls], &S.h_jobs[k].G, sizeof(Globals)) != 0) {
        uni_scene[cls] = -1;
      }
    }
  }
  S.h_ctl[0].total_tasks = (unsigned long long)tb;             // all jobs (frames)
  S.h_ctl[0].njobs = (int)plan.size();
  const bool frames = S.o.frames_every > 0;
  auto minb_of = [&](int grp) {
    (void)grp;
    return S.o.occupancy > 0 ? std::min(S.o.occupancy, 4) : batch_minb(grp > 4 ? grp - 4 : grp, grp > 4);
  };
  auto launch_group = [&](int grp) {
    const int cls = grp > 4 ? grp - 4 : grp;
    BatchUniform u;
    const bool uniform = uni_scene[grp] >= 0;
    if (uniform) {
      u.S = S.scenes[uni_scene[grp]]->view;
      u.G = uni_G[grp];
    }
    int stack = 0;
    for (const auto &pl : plan)
      if (pl.cls == grp) stack = std::max(stack, S.scenes[S.jobs[pl.id].req.scene]->view.short_stack);
    launch_batch(cls, minb_of(grp), grp > 4, S.st, S.d_jobs, S.d_ctl + grp, S.sms, uniform ? &u : nullptr, stack);
  };
  auto kernels = [&](bool all_groups) {
    for (int c = 1; c < RB_GROUPS; ++c)
      if (all_groups || S.h_ctl[c].njobs > 0) launch_group(c);
  };
  // wavefront jobs: one engine run per scene over its planned jobs
  uint64_t wf_paths = 0, wf_segments = 0;
  auto run_wavefront = [&]() -> int {
    std::vector<int> scenes;
    for (size_t k : wf_k) {
      const int sc = S.jobs[plan[k].id].req.scene;
      if (std::find(scenes.begin(), scenes.end(), sc) == scenes.end()) scenes.push_back(sc);
    }
    for (int sc : scenes) {
      std::vector<WfJob> wj;
      for (size_t k : wf_k) {
        const Job &J = S.jobs[plan[k].id];
        if (J.req.scene != sc) continue;
        WfJob w;
        std::memset(&w, 0, sizeof w);
        w.P = S.h_jobs[k].P;
        w.G = S.h_jobs[k].G;
        w.acc = J.acc64;
        wj.push_back(w);
      }
      uint64_t c[4] = {0, 0, 0, 0};
      const int rc = wf_render_jobs(S.scenes[sc], wj.data(), (int)wj.size(), S.wf_cap, c, S.st_wf);
      if (rc != RB_OK) return rc;
      wf_segments += c[0];
      wf_paths += c[1];
    }
    return RB_OK;
  };
  const long long frame_blocks_cap = (S.o.paths_per_iteration + 255) / 256 + 1;
  auto run_per_frame = [&]() -> int {
    int used = 0, rc = RB_OK;
    for (size_t i = 0; i < pf_k.size() && rc == RB_OK; ++i) {
      const size_t k = pf_k[i];
      const Job &J = S.jobs[plan[k].id];
      const BatchJob &B = S.h_jobs[k];
      const int n = J.req.width * J.req.height;
      cudaStream_t ps = S.st_pf[i % RB_PF_STREAMS];
      if (i < RB_PF_STREAMS) {
        cudaStreamWaitEvent(ps, S.ev_pf_fork, 0);
        ++used;
      }
      rc = launch_render(S.scenes[J.req.scene], B.G, B.P, J.acc, J.acc + n, nullptr, S.d_pfc, ps);
    }
    for (int q = 0; q < used; ++q) {  // join, also after an error
      cudaEventRecord(S.ev_pf_join[q], S.st_pf[q]);
      cudaStreamWaitEvent(S.st, S.ev_pf_join[q], 0);
    }
    return rc;
  };
  if (S.o.use_graph && wf_k.empty() && pf_k.empty() && !(frames && (tb + 255) / 256 > frame_blocks_cap)) {
    // One graph, reused every iteration: table and control blocks are copied
    // from pinned staging when the graph runs, the three class kernels are
    // persistent (grid = resident blocks) and exit at once when their class
    // has no work this iteration.
    bool same_uniform = true;
    for (int c = 1; c < RB_GROUPS; ++c)
      same_uniform = same_uniform && uni_scene[c] == S.graph_scene[c] &&
                     std::memcmp(&uni_G[c], &S.graph_G[c], sizeof(Globals)) == 0;
    if (!S.graph || S.graph_frames != (int)frames || !same_uniform) {
      if (S.graph) cudaGraphExecDestroy(S.graph);
      S.graph = nullptr;
      cudaGraph_t g;
      if (!cuda_ok(cudaStreamBeginCapture(S.st, cudaStreamCaptureModeThreadLocal), "graph capture")) return RB_ERR_CUDA;
      cudaMemcpyAsync(S.d_jobs, S.h_jobs, sizeof(BatchJob) * S.o.max_active_jobs, cudaMemcpyHostToDevice, S.st);
      cudaMemcpyAsync(S.d_ctl, S.h_ctl, sizeof(BatchCtl) * RB_GROUPS, cudaMemcpyHostToDevice, S.st);
      kernels(true);
      if (frames) k_batch_frames<<<(unsigned)frame_blocks_cap, 256, 0, S.st>>>(S.d_jobs, S.d_ctl);
      if (!cuda_ok(cudaStreamEndCapture(S.st, &g), "graph capture")) return RB_ERR_CUDA;
      if (!cuda_ok(cudaGraphInstantiate(&S.graph, g, 0), "graph instantiate")) return RB_ERR_CUDA;
      cudaGraphDestroy(g);
      S.graph_frames = (int)frames;
      for (int c = 0; c < RB_GROUPS; ++c) {
        S.graph_scene[c] = uni_scene[c];
        S.graph_G[c] = uni_G[c];
      }
    }
    cudaEventRecord(S.ev0, S.st);  // after any capture/instantiation: device time only
    if (!cuda_ok(cudaGraphLaunch(S.graph, S.st), "graph launch")) return RB_ERR_CUDA;
    g_launches += (RB_GROUPS - 1) + (frames ? 1 : 0);
  } else {
    cudaEventRecord(S.ev0, S.st);
    cudaMemcpyAsync(S.d_jobs, S.h_jobs, sizeof(BatchJob) * plan.size(), cudaMemcpyHostToDevice, S.st);
    cudaMemcpyAsync(S.d_ctl, S.h_ctl, sizeof(BatchCtl) * RB_GROUPS, cudaMemcpyHostToDevice, S.st);
    cudaEventRecord(S.ev_up, S.st);
    if (!pf_k.empty()) {
      cudaMemsetAsync(S.d_pfc, 0, sizeof(unsigned long long) * 4, S.st);
      cudaEventRecord(S.ev_pf_fork, S.st);
    }
    kernels(false);
    if (!pf_k.empty()) {
      const int rc = run_per_frame();
      if (rc != RB_OK) return rc;
      cudaMemcpyAsync(S.h_pfc, S.d_pfc, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, S.st);
    }
    if (!wf_k.empty()) {
      // the wavefront jobs touch only their own sums, so they start after the
      // uploads and run beside the class kernels (their blocks take the SMs
      // the class kernels' tails leave idle); the iteration ends after both
      cudaStreamWaitEvent(S.st_wf, S.ev_up, 0);
      const int rc = run_wavefront();
      cudaEventRecord(S.ev_wf, S.st_wf);
      cudaStreamWaitEvent(S.st, S.ev_wf, 0);
      if (rc != RB_OK) return rc;
    }
    if (frames) {
      k_batch_frames<<<(unsigned)((tb + 255) / 256), 256, 0, S.st>>>(S.d_jobs, S.d_ctl);
      g_launches++;
    }
  }
  cudaEventRecord(S.ev1, S.st);
  cudaMemcpyAsync(S.h_ctl, S.d_ctl, sizeof(BatchCtl) * RB_GROUPS, cudaMemcpyDeviceToHost, S.st);
  if (!cuda_ok(cudaStreamSynchronize(S.st), "batched iteration")) return RB_ERR_CUDA;
  float ms_it = 0.f;
  cudaEventElapsedTime(&ms_it, S.ev0, S.ev1);
  S.stats.device_seconds += ms_it * 1e-3;
  S.last_ms = ms_it;
  // latency-target controller: the quantum follows the measured iteration time
  // (only when the iteration used its whole quantum; a short queue says nothing)
  if (S.o.target_iteration_ms > 0.0f && ms_it > 0.0f && budget <= 0) {
    const double scale = std::min(2.0, std::max(0.5, (double)S.o.target_iteration_ms / (double)ms_it));
    const int64_t q = (int64_t)std::llround((double)S.quantum * scale);
    S.quantum = std::min<int64_t>(S.o.paths_per_iteration, std::max<int64_t>(int64_t(1) << 18, q));
  }
  S.stats.iterations++;
  for (int c = 1; c < RB_GROUPS; ++c) {
    S.stats.paths += (int64_t)S.h_ctl[c].paths;
    S.stats.segments += (int64_t)S.h_ctl[c].segments;
  }
  S.stats.paths += (int64_t)wf_paths;
  S.stats.segments += (int64_t)wf_segments;
  if (!pf_k.empty()) {
    S.stats.segments += (int64_t)S.h_pfc[0];
    S.stats.paths += (int64_t)S.h_pfc[1];
  }
  if (frames) S.stats.frames += (int64_t)plan.size();
  // per-job convergence of the jobs that asked for it
  {
    std::vector<size_t> conv_k;
    for (size_t k = 0; k < plan.size(); ++k)
      if (S.jobs[plan[k].id].req.converge_threshold > 0.0f) conv_k.push_back(k);
    if (!conv_k.empty()) {
      cudaMemsetAsync(S.d_conv, 0, sizeof(unsigned long long) * conv_k.size(), S.st);
      for (size_t c = 0; c < conv_k.size(); ++c) {
        Job &J = S.jobs[plan[conv_k[c]].id];
        const int n = J.req.width * J.req.height;
        const int spp_now = J.spp_done + plan[conv_k[c]].spp;
        const int checked = J.spp_done > 0 && spp_now >= J.req.converge_min_spp ? 1 : 0;
        k_job_converge<<<(n + 255) / 256, 256, 0, S.st>>>(J.acc, J.acc64, J.lum, n, spp_now, checked,
                                                          J.req.converge_threshold, S.d_conv + c);
        g_launches++;
      }
      cudaMemcpyAsync(S.h_conv, S.d_conv, sizeof(unsigned long long) * conv_k.size(), cudaMemcpyDeviceToHost,
                      S.st);
      if (!cuda_ok(cudaStreamSynchronize(S.st), "job convergence")) return RB_ERR_CUDA;
      for (size_t c = 0; c < conv_k.size(); ++c) {
        Job &J = S.jobs[plan[conv_k[c]].id];
        const double n = (double)J.req.width * J.req.height;
        if ((double)S.h_conv[c] >= (double)J.req.converge_fraction * n) J.converged = true;
      }
    }
  }
  // retire
  const double t = S.now();
  std::vector<int64_t> still;
  std::unordered_map<int64_t, int> got;
  for (const Plan &p : plan) got[p.id] = p.spp;
  for (int64_t id : S.active) {
    Job &J = S.jobs[id];
    auto it = got.find(id);
    if (it != got.end()) J.spp_done += it->second;
    if (J.spp_done >= J.req.spp || J.converged) {
      J.state = 2;
      J.t_done = t;
      S.stats.jobs_done++;
      S.latencies.push_back(J.t_done - J.t_arrival);
      S.last_done = t;
    } else {
      still.push_back(id);
    }
  }
  S.active.swap(still);
  return (int)(S.active.size() + S.queue.size());
}

}  // namespace rb

using namespace rb;

struct rb_server {
  Server s;
};

extern "C" {

void rb_job_default(rb_job_request *r) {
  if (!r) return;
  std::memset(r, 0, sizeof *r);
  r->max_depth = 16;
  r->spp = 1;
  r->light_intensity = 1.0f;
  r->background_intensity = 1.0f;
  r->metal_fuzziness = 0.8f;
  r->glass_ior = 1.5f;
  r->dof_aperture = 0.1f;
  r->dof_focus = 10.0f;
  r->converge_min_spp = 32;    // the reference's min_adaptive_samples default
  r->converge_fraction = 1.0f;
}

void rb_server_default_opts(rb_server_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->memory_budget_bytes = (int64_t)150 << 30;
  o->max_active_jobs = 256;
  o->paths_per_iteration = 64ll << 20;
  o->max_spp_per_iteration = 64;
  o->use_graph = 1;
  o->frames_every = 0;
  o->wavefront_field = 1;
  // diffuse and classic scenes on the per-frame kernel: measured on 200 jobs of
  // the serving mix, served Cornell 9769 -> 12277 Mpaths/s and One-Weekend
  // 3501 -> 4069; the full class (icospheres) stays on the batched kernel
  // (3948 there against 3026 per frame)
  o->per_frame_classes = (1 << RB_MS_DIFFUSE) | (1 << RB_MS_CLASSIC);
}

rb_server *rb_server_create(const rb_server_opts *opts, void *stream) {
  rb_server *r = new rb_server();
  Server &S = r->s;
  rb_server_default_opts(&S.o);
  if (opts) S.o = *opts;
  if (S.o.max_active_jobs <= 0 || S.o.max_active_jobs > 1024 || S.o.paths_per_iteration <= 0 ||
      S.o.max_spp_per_iteration <= 0 || S.o.memory_budget_bytes <= 0) {
    set_error("rb_server_create: invalid options");
    delete r;
    return nullptr;
  }
  S.st = static_cast<cudaStream_t>(stream);
  if (!S.st) {
    cudaStreamCreateWithFlags(&S.st, cudaStreamNonBlocking);
    S.own_stream = true;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&S.sms, cudaDevAttrMultiProcessorCount, dev);
  bool ok = cuda_ok(cudaMallocHost(&S.h_jobs, sizeof(BatchJob) * S.o.max_active_jobs), "server pinned jobs") &&
            cuda_ok(cudaMalloc(&S.d_jobs, sizeof(BatchJob) * S.o.max_active_jobs), "server jobs") &&
            cuda_ok(cudaMallocHost(&S.h_ctl, sizeof(BatchCtl) * RB_GROUPS), "server pinned ctl") &&
            cuda_ok(cudaMalloc(&S.d_ctl, sizeof(BatchCtl) * RB_GROUPS), "server ctl") &&
            cuda_ok(cudaMallocHost(&S.h_conv, sizeof(unsigned long long) * S.o.max_active_jobs), "server conv") &&
            cuda_ok(cudaMalloc(&S.d_conv, sizeof(unsigned long long) * S.o.max_active_jobs), "server conv") &&
            cuda_ok(cudaMallocHost(&S.h_pfc, sizeof(unsigned long long) * 4), "server per-frame counters") &&
            cuda_ok(cudaMalloc(&S.d_pfc, sizeof(unsigned long long) * 4), "server per-frame counters");
  if (!ok) {
    rb_server_destroy(r);
    return nullptr;
  }
  std::memset(S.h_jobs, 0, sizeof(BatchJob) * S.o.max_active_jobs);
  preload_batch_kernels();
  for (int c = 0; c < RB_GROUPS; ++c) {
    S.graph_scene[c] = -1;
    std::memset(&S.graph_G[c], 0, sizeof(Globals));
  }
  cudaEventCreate(&S.ev0);
  cudaEventCreate(&S.ev1);
  {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (!cuda_ok(cudaMemPoolCreate(&S.pool, &props), "server job pool")) {
      S.pool = nullptr;
      rb_server_destroy(r);
      return nullptr;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(S.pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  bool streams_ok = cuda_ok(cudaStreamCreateWithFlags(&S.st_wf, cudaStreamNonBlocking), "server wavefront stream") &&
                    cuda_ok(cudaEventCreateWithFlags(&S.ev_up, cudaEventDisableTiming), "server event") &&
                    cuda_ok(cudaEventCreateWithFlags(&S.ev_wf, cudaEventDisableTiming), "server event") &&
                    cuda_ok(cudaEventCreateWithFlags(&S.ev_pf_fork, cudaEventDisableTiming), "server event");
  for (int q = 0; q < RB_PF_STREAMS && streams_ok; ++q)
    streams_ok = cuda_ok(cudaStreamCreateWithFlags(&S.st_pf[q], cudaStreamNonBlocking), "server per-frame stream") &&
                 cuda_ok(cudaEventCreateWithFlags(&S.ev_pf_join[q], cudaEventDisableTiming), "server event");
  if (!streams_ok) {
    rb_server_destroy(r);
    return nullptr;
  }
  std::memset(&S.stats, 0, sizeof S.stats);
  S.quantum = S.o.paths_per_iteration;
  S.t0 = std::chrono::steady_clock::now();
  return r;
}

void rb_server_destroy(rb_server *r) {
  if (!r) return;
  Server &S = r->s;
  if (S.st) cudaStreamSynchronize(S.st);
  for (auto &kv : S.jobs) free_job(S, kv.second);
  if (S.st) cudaStreamSynchronize(S.st);
  if (S.graph) cudaGraphExecDestroy(S.graph);
  if (S.h_jobs) cudaFreeHost(S.h_jobs);
  if (S.d_jobs) cudaFree(S.d_jobs);
  if (S.h_ctl) cudaFreeHost(S.h_ctl);
  if (S.d_ctl) cudaFree(S.d_ctl);
  if (S.h_conv) cudaFreeHost(S.h_conv);
  if (S.d_conv) cudaFree(S.d_conv);
  if (S.h_pfc) cudaFreeHost(S.h_pfc);
  if (S.d_pfc) cudaFree(S.d_pfc);
  if (S.ev0) cudaEventDestroy(S.ev0);
  if (S.ev1) cudaEventDestroy(S.ev1);
  if (S.st_wf) {
    cudaStreamSynchronize(S.st_wf);
    cudaStreamDestroy(S.st_wf);
  }
  if (S.ev_up) cudaEventDestroy(S.ev_up);
  if (S.ev_wf) cudaEventDestroy(S.ev_wf);
  for (int q = 0; q < RB_PF_STREAMS; ++q) {
    if (S.st_pf[q]) {
      cudaStreamSynchronize(S.st_pf[q]);
      cudaStreamDestroy(S.st_pf[q]);
    }
    if (S.ev_pf_join[q]) cudaEventDestroy(S.ev_pf_join[q]);
  }
  if (S.ev_pf_fork) cudaEventDestroy(S.ev_pf_fork);
  if (S.pool) {
    if (S.st) cudaStreamSynchronize(S.st);  // the jobs' stream-ordered frees have run
    cudaMemPoolDestroy(S.pool);
  }
  if (S.own_stream && S.st) cudaStreamDestroy(S.st);
  delete r;
}

int rb_server_add_scene(rb_server *r, const rb_cuda_scene *scene) {
  if (!r) return RB_ERR_INVALID_ARG;
  const DeviceScene *ds = lookup_scene(scene);
  if (!ds) {
    set_error("rb_server_add_scene: unknown scene handle");
    return RB_ERR_NOT_FOUND;
  }
  // the wavefront engine's queues and march buffers are allocated when a
  // smooth-SDF scene joins, not inside the first request's iteration
  if (on_wavefront_scene(r->s, ds)) {
    r->s.wf_cap = std::max(r->s.wf_cap, scene_wf_queue(ds));
    const int rc = wf_render_jobs(ds, nullptr, 0, r->s.wf_cap, nullptr, r->s.st);
    if (rc != RB_OK) return rc;
  }
  r->s.scenes.push_back(ds);
  return (int)r->s.scenes.size() - 1;
}

int64_t rb_server_submit(rb_server *r, const rb_job_request *q) {
  if (!r || !q) return RB_ERR_INVALID_ARG;
  Server &S = r->s;
  if (q->scene < 0 || q->scene >= (int)S.scenes.size() || q->width <= 0 || q->height <= 0 || q->spp <= 0 ||
      q->max_depth < 0 || (int64_t)q->width * q->height > (1ll << 31) - 1 ||
      (q->converge_threshold > 0.0f && !(q->converge_fraction > 0.0f && q->converge_fraction <= 1.0f))) {
    set_error("rb_server_submit: invalid request");
    return RB_ERR_INVALID_ARG;
  }
  Job J;
  J.req = *q;
  J.id = S.next_id++;
  J.t_arrival = S.now();
  if (S.first_arrival < 0) S.first_arrival = J.t_arrival;
  S.jobs.emplace(J.id, J);
  S.queue.push_back(J.id);
  return J.id;
}

int rb_server_step(rb_server *r) {
  if (!r) return RB_ERR_INVALID_ARG;
  return server_step(r->s);
}

int rb_server_job_status(rb_server *r, int64_t id, rb_job_status *out) {
  if (!r || !out) return RB_ERR_INVALID_ARG;
  auto it = r->s.jobs.find(id);
  if (it == r->s.jobs.end()) return RB_ERR_NOT_FOUND;
  const Job &J = it->second;
  out->state = J.state;
  out->spp_done = J.spp_done;
  out->t_arrival = J.t_arrival;
  out->t_admit = J.t_admit;
  out->t_done = J.t_done;
  out->device_bytes = J.bytes;
  out->error = J.error;
  out->reserved_ = 0;
  return RB_OK;
}

int rb_server_fetch(rb_server *r, int64_t id, float *rgb, uint8_t *frame) {
  if (!r) return RB_ERR_INVALID_ARG;
  Server &S = r->s;
  auto it = S.jobs.find(id);
  if (it == S.jobs.end()) return RB_ERR_NOT_FOUND;
  Job &J = it->second;
  if (!J.acc && !J.acc64) {
    set_error("rb_server_fetch: job has no device buffers (queued, rejected or released)");
    return RB_ERR_STATE;
  }
  cudaStreamSynchronize(S.st);
  const int64_t n = (int64_t)J.req.width * J.req.height;
  if (rgb) {
    if (J.acc64) {
      std::vector<double> h(n * 4);
      if (!cuda_ok(cudaMemcpy(h.data(), J.acc64, n * 32, cudaMemcpyDeviceToHost), "fetch")) return RB_ERR_CUDA;
      for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) rgb[3 * i + k] = (float)h[4 * i + k];
    } else {
      std::vector<float> h(n * 8);
      if (!cuda_ok(cudaMemcpy(h.data(), J.acc, n * 32, cudaMemcpyDeviceToHost), "fetch")) return RB_ERR_CUDA;
      for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) rgb[3 * i + k] = (float)((double)h[4 * i + k] - (double)h[4 * (n + i) + k]);
    }
  }
  if (frame) {
    if (!J.frame) {
      set_error("rb_server_fetch: frames are off (rb_server_opts.frames_every = 0)");
      return RB_ERR_STATE;
    }
    if (!cuda_ok(cudaMemcpy(frame, J.frame, n * 4, cudaMemcpyDeviceToHost), "fetch frame")) return RB_ERR_CUDA;
  }
  return RB_OK;
}

int rb_server_release(rb_server *r, int64_t id) {
  if (!r) return RB_ERR_INVALID_ARG;
  auto it = r->s.jobs.find(id);
  if (it == r->s.jobs.end()) return RB_ERR_NOT_FOUND;
  if (it->second.state == 1) {
    set_error("rb_server_release: job is still active");
    return RB_ERR_STATE;
  }
  free_job(r->s, it->second);
  return RB_OK;
}

int rb_server_run_trace(rb_server *r, const rb_job_request *reqs, int64_t n, int realtime, int keep, double *lat) {
  if (!r || (!reqs && n > 0) || n < 0) return RB_ERR_INVALID_ARG;
  Server &S = r->s;
  std::vector<int64_t> ids(n, -1);
  std::vector<int64_t> order(n);
  for (int64_t i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int64_t a, int64_t b) { return reqs[a].arrival_time < reqs[b].arrival_time; });
  const double base = S.now();
  int64_t next = 0;
  std::vector<char> released(n, 0);
  while (true) {
    const double t = S.now() - base;
    while (next < n && (!realtime || reqs[order[next]].arrival_time <= t)) {
      const int64_t k = order[next];
      const int64_t id = rb_server_submit(r, &reqs[k]);
      if (id < 0) return (int)id;
      if (realtime) S.jobs[id].t_arrival = base + reqs[k].arrival_time;  // nominal arrival
      ids[k] = id;
      ++next;
    }
    const int left = server_step(S);
    if (left < 0) return left;
    if (!keep)
      for (int64_t k = 0; k < n; ++k)
        if (ids[k] >= 0 && !released[k] && S.jobs[ids[k]].state == 2) {
          free_job(S, S.jobs[ids[k]]);
          released[k] = 1;
        }
    if (left == 0 && next >= n) break;
    if (left == 0 && realtime && next < n) {
      // idle until the next arrival
      const double wait = reqs[order[next]].arrival_time - (S.now() - base);
      if (wait > 0) {
        auto until = std::chrono::steady_clock::now() + std::chrono::duration<double>(wait);
        while (std::chrono::steady_clock::now() < until) {
        }
      }
    }
  }
  if (lat)
    for (int64_t k = 0; k < n; ++k) {
      const Job &J = S.jobs[ids[k]];
      lat[k] = J.state == 2 ? J.t_done - J.t_arrival : -1.0;
    }
  return RB_OK;
}

int rb_server_get_stats(rb_server *r, rb_server_stats *out) {
  if (!r || !out) return RB_ERR_INVALID_ARG;
  Server &S = r->s;
  *out = S.stats;
  out->peak_device_bytes = S.peak_bytes;
  out->quantum_paths = S.quantum;
  out->last_iteration_ms = S.last_ms;
  out->wall_seconds = S.first_arrival >= 0 ? S.last_done - S.first_arrival : 0.0;
  std::vector<double> l = S.latencies;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto q = [&](double p) {
      const double idx = p * (l.size() - 1);
      const size_t i = (size_t)idx;
      const double f = idx - i;
      return i + 1 < l.size() ? l[i] * (1 - f) + l[i + 1] * f : l[i];
    };
    out->p50_latency = q(0.5);
    out->p99_latency = q(0.99);
    double sum = 0;
    for (double v : l) sum += v;
    out->mean_latency = sum / l.size();
  }
  return RB_OK;
}


// ---------------------------------------------------------------------------
// Several views of one scene in one persistent launch
// ---------------------------------------------------------------------------
}  // extern "C"

namespace rb {
namespace {
// Per-device job table: pinned staging, device copy, and an event that marks
// the staging buffer free again (its last upload has run).
struct ViewsTable {
  unsigned char *h = nullptr, *d = nullptr;
  size_t cap = 0;
  cudaEvent_t uploaded = nullptr;  // staging buffer free again
  cudaEvent_t consumed = nullptr;  // device table free again (its launch has run)
};
std::mutex g_views_mu;
ViewsTable g_views[64];
}  // namespace
}  // namespace rb

extern "C" {

int rb_render_views(const rb_cuda_scene *scene, int n_views, int width, int height, const double *frames, int samples,
                    int sample_base, int max_depth, float *accum, uint64_t *counters, void *stream) {
  DeviceScene *ds = lookup_scene(scene);
  if (!ds) {
    set_error("rb_render_views: unknown scene handle");
    return RB_ERR_NOT_FOUND;
  }
  if (n_views <= 0 || n_views > 4096 || width <= 0 || height <= 0 || !frames || !accum || samples < 0 ||
      max_depth < 0 || sample_base < 0 || (long long)width * height * n_views > (1ll << 40)) {
    set_error("rb_render_views: invalid argument");
    return RB_ERR_INVALID_ARG;
  }
  if (samples == 0) return RB_OK;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) {
    set_error("rb_render_views: device ordinal out of range");
    return RB_ERR_INVALID_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> lock(g_views_mu);
  ViewsTable &T = g_views[dev];
  const size_t bytes = sizeof(BatchCtl) + sizeof(BatchJob) * (size_t)n_views;
  if (T.uploaded) cudaEventSynchronize(T.uploaded);  // the previous upload has left the staging buffer
  if (bytes > T.cap) {
    if (T.d) cudaFree(T.d);
    if (T.h) cudaFreeHost(T.h);
    T.d = T.h = nullptr;
    T.cap = 0;
    if (!cuda_ok(cudaMalloc(&T.d, bytes), "rb_render_views: job table") ||
        !cuda_ok(cudaMallocHost(&T.h, bytes), "rb_render_views: pinned job table"))
      return RB_ERR_CUDA;
    T.cap = bytes;
  }
  if (!T.uploaded && !cuda_ok(cudaEventCreateWithFlags(&T.uploaded, cudaEventDisableTiming), "rb_render_views: event"))
    return RB_ERR_CUDA;
  if (!T.consumed && !cuda_ok(cudaEventCreateWithFlags(&T.consumed, cudaEventDisableTiming), "rb_render_views: event"))
    return RB_ERR_CUDA;
  BatchCtl *ctl = reinterpret_cast<BatchCtl *>(T.h);
  BatchJob *jobs = reinterpret_cast<BatchJob *>(T.h + sizeof(BatchCtl));
  std::memset(T.h, 0, bytes);
  const Globals G = current_globals();
  const uint32_t seed = current_opts().seed;
  const long long px = (long long)width * height;
  for (int v = 0; v < n_views; ++v) {
    BatchJob &B = jobs[v];
    B.S = ds->view;
    B.P = frame_from(frames + 21 * (size_t)v, width, height);
    B.P.samples = samples;
    B.P.sample_base = sample_base;
    B.P.max_depth = max_depth;
    B.P.seed = seed;
    B.P.salt = (uint32_t)v;  // view 0 draws the streams of rb_render_accumulate
    B.G = G;
    B.acc = reinterpret_cast<float4 *>(accum) + 2 * px * v;
    B.task_begin = px * v;
    B.spp_total = sample_base + samples;
  }
  ctl->total_tasks = (unsigned long long)(px * n_views);
  ctl->njobs = n_views;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // a previous call's launch (possibly on another stream) must be done with the device table
  if (!cuda_ok(cudaStreamWaitEvent(st, T.consumed, 0), "rb_render_views: wait") ||
      !cuda_ok(cudaMemcpyAsync(T.d, T.h, bytes, cudaMemcpyHostToDevice, st), "rb_render_views: upload") ||
      !cuda_ok(cudaEventRecord(T.uploaded, st), "rb_render_views: event"))
    return RB_ERR_CUDA;
  const rb_render_opts o = current_opts();
  const int minb = o.reserved[0] > 0 ? std::min(o.reserved[0], 4) : batch_minb(ds->ms, G.nee != 0);
  BatchCtl *d_ctl = reinterpret_cast<BatchCtl *>(T.d);
  BatchUniform uni;  // every view shares the scene and the settings
  uni.S = ds->view;
  uni.G = G;
  launch_batch(ds->ms, minb, G.nee != 0, st, reinterpret_cast<const BatchJob *>(T.d + sizeof(BatchCtl)), d_ctl, sms,
               &uni, ds->view.short_stack);
  if (!cuda_ok(cudaGetLastError(), "rb_render_views: launch")) return RB_ERR_CUDA;
  if (counters &&
      !cuda_ok(cudaMemcpyAsync(counters, &d_ctl->segments, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st),
               "rb_render_views: counters"))
    return RB_ERR_CUDA;
  return cuda_ok(cudaEventRecord(T.consumed, st), "rb_render_views: event") ? RB_OK : RB_ERR_CUDA;
}

}  // extern "C"
