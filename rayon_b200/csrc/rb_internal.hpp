// Internal declarations shared by the translation units of the library.
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "../../include/rayon_b200.h"
#include "rb_shade.cuh"

namespace rb {

inline float __int_as_float_host(int i) {
  float f;
  std::memcpy(&f, &i, 4);
  return f;
}
inline float __uint_as_float_host(uint32_t i) {
  float f;
  std::memcpy(&f, &i, 4);
  return f;
}
inline uint32_t __float_as_uint_host(float f) {
  uint32_t i;
  std::memcpy(&i, &f, 4);
  return i;
}

// Allocator that leaves elements uninitialised on a value-less resize, so a
// large host array is first touched (and its pages faulted in) by the threads
// that fill it rather than by one thread zeroing it.
template <class T>
struct uninit_alloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = uninit_alloc<U>;
  };
  uninit_alloc() = default;
  template <class U>
  uninit_alloc(const uninit_alloc<U> &) noexcept {}
  template <class U>
  void construct(U *) noexcept {}
  template <class U, class... A>
  void construct(U *p, A &&...a) {
    ::new ((void *)p) U(std::forward<A>(a)...);
  }
};

// Device layout assembled on the host before upload.
struct HostLayout {
  std::vector<float4, uninit_alloc<float4>> nodes;  // 4 per interior node, every word written
  std::vector<rbd::QNode> qnodes;     // quantised copy of nodes
  std::vector<float4> wnodes;         // 4-wide copy of nodes (8 per wide node) or empty
  std::vector<float4, uninit_alloc<float4>> prims;  // 3 per primitive, zeroed record by record
  std::vector<float4> normals;        // 3 per primitive (vertex normals) or empty
  std::vector<rbd::DevMaterial> mats;
  std::vector<rbd::LightRec> lights;
  std::vector<rbd::SdfPrim> sdf;
  std::vector<float4> groups;         // grouped linear layout: 2 per group
  int root_ref = 0;
  int wide_root = 0;                  // root of wnodes (a leaf ref when the root is a leaf)
  float root_box[6] = {0, 0, 0, 0, 0, 0};
  float light_area = 0.0f;
  bool use_bvh = false;
  int ms = 3;  // kernel material class
};

struct DeviceScene {
  rbd::SceneView view;
  void *handle = nullptr;  // device pointer handed out as CudaScene::Scene*
  size_t bytes = 0;
  int ms = 3;
  int layout_kind = 0, layout_leaf = 0;
  float probe_ms = 0.0f;
  // launch configuration chosen by the autotuner (0: the class defaults)
  int tuned_minb = 0, tuned_bx = 0, tuned_by = 0;
  int tuned_fetch = 0;  // k_render schedule: 0 default (fetch), 1 grid, 2 fetch
  int wf_queue = 0;          // wavefront engine path slots for this scene (0: default)
  bool tune_cached = false;  // the decision came from the per-(GPU, scene) cache
};

// FP32 camera frame for the kernels (cast from the FP64 frame, as
// renderer_cuda_device.cu:279-284 casts its double arguments).
struct FrameF {
  rbd::f3 center, p00, du, dv, cu, cv;
  int width, height, samples, sample_base, max_depth;
  uint32_t seed, salt;
  int min_adaptive;
  float adaptive_threshold;
};

// One job of a wavefront-engine run: its camera frame (P.samples samples per
// pixel from P.sample_base, P.max_depth, stream seed and salt), shading
// settings, FP64 accumulation (w*h*4 doubles: xyz sums, pad) and its first
// work item (set by wf_render_jobs). Work items are job-major, then
// sample-major within the job.
struct __align__(16) WfJob {
  FrameF P;
  rbd::Globals G;
  double *acc;
  unsigned long long item_begin;
};

struct DeviceScene;
// Renders the jobs (host table) of one scene on the wavefront engine until
// every path has ended, ordered after and before `caller`. counters (host,
// may be null): segments, paths, stack overflows, iterations.
int wf_render_jobs(const DeviceScene *ds, WfJob *jobs, int njobs, int queue_capacity, uint64_t *counters,
                   cudaStream_t caller);

bool cuda_ok(cudaError_t e, const char *what);
void set_error(const std::string &msg);

// Host-side fault injection (rb_inject_alloc_failures): the next n device
// allocations at a site fail as if the device were out of memory. Consumes
// one pending failure and returns true when the allocation must fail.
enum AllocSite { RB_SITE_SERVER_JOB = 0, RB_SITE_WAVEFRONT = 1, RB_SITE_COUNT = 2 };
bool injected_alloc_failure(int site);
DeviceScene *lookup_scene(const void *handle);
void build_quantized(HostLayout &L);
// Fills L.wnodes / L.wide_root from the binary nodes (wide_bvh.cu).
void build_wide(HostLayout &L);
FrameF frame_from(const double *fr, int w, int h);
// The per-frame kernel over one frame's sample range (rb_render.cu).
int launch_render(const DeviceScene *ds, const rbd::Globals &G, const FrameF &P, float4 *acc, float4 *comp,
                  int *counts, unsigned long long *counters, cudaStream_t st);
struct HostScene;
rbd::Globals current_globals();
rb_render_opts current_opts();

}  // namespace rb
