// Device scene upload, the per-frame render kernels and the drop-in C-ABI
// (renderer_cuda_device.cuh:8-67) of the B200 render path.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "host_scene.hpp"
#include "rb_internal.hpp"
#include "rb_path.cuh"
#include "rb_render_kernel.cuh"

using namespace rbd;

namespace rb {

const HostScene &host_scene_of(const rb_scene_desc *s);

std::atomic<unsigned long long> g_launches{0};

// ---------------------------------------------------------------------------
// Registries (host side)
// ---------------------------------------------------------------------------
static std::mutex g_mu;
static std::unordered_map<const void *, DeviceScene *> g_scenes;   // handle -> scene
static std::unordered_map<const void *, size_t> g_accum_bytes;      // accum allocations
static std::unordered_map<const void *, uint32_t> g_rng_ctx;        // samples already drawn

bool cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}

DeviceScene *lookup_scene(const void *handle) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_scenes.find(handle);
  return it == g_scenes.end() ? nullptr : it->second;
}

// Reference __constant__ defaults (renderer_cuda_device.cu:18-26).
static Globals g_globals = {1.0f, 1.0f, 0.8f, 1.5f, 0, 0.1f, 10.0f, 0};
static rb_render_opts g_opts = {0, 1, 0x5EEDu, 0, 0, {0, 0, 0, 0}};
Globals current_globals() {
  Globals g = g_globals;
  g.nee = g_opts.nee;
  return g;
}
rb_render_opts current_opts() { return g_opts; }

// ---------------------------------------------------------------------------
// Host -> device layout
// ---------------------------------------------------------------------------
static float ftz_sub(float a, float b) {
  float r = a - b;
  if (std::fabs(r) < 1.17549435e-38f) r = std::copysign(0.0f, r);
  return r;
}

static DevMaterial resolve_material(const rb_material_desc &d) {
  // apply_material (cuda_raytracer.cuh:418-485), resolved once per material.
  DevMaterial m;
  std::memset(&m, 0, sizeof m);
  auto f = [](const double *v) { return f3((float)v[0], (float)v[1], (float)v[2]); };
  const f3 albedo = f(d.albedo);
  m.color = albedo;
  m.emission = f(d.emission);
  m.eta = f(d.eta);
  m.k = f(d.k);
  m.roughness = d.roughness;
  m.ior = d.refractive_index;
  m.anisotropy = d.anisotropy;
  m.film_thickness = d.film_thickness;
  m.film_ior = d.film_ior;
  m.pattern = d.pattern == 1 ? 1 : 0;  // FIBONACCI_DOTS; other patterns fall to the base colour
  m.pattern_color = f(d.pattern_color);
  m.pattern_p1 = d.pattern_param1;
  m.pattern_p2 = d.pattern_param2;
  switch (d.type) {
    case RB_MAT_LAMBERTIAN: m.kind = L_LAMBERTIAN; break;
    case RB_MAT_MIRROR: m.kind = L_MIRROR; break;
    case RB_MAT_METAL:
    case RB_MAT_ROUGH_MIRROR:
      m.kind = L_ROUGH_MIRROR;
      m.roughness = d.roughness > 0.0f ? d.roughness : 0.3f;
      break;
    case RB_MAT_GLASS:
    case RB_MAT_DIELECTRIC: m.kind = L_GLASS; break;
    case RB_MAT_LIGHT: m.kind = L_LIGHT; break;
    case RB_MAT_CONSTANT: m.kind = L_CONSTANT; break;
    case RB_MAT_SHOW_NORMALS: m.kind = L_SHOW_NORMALS; break;
    case RB_MAT_ANISOTROPIC_METAL: m.kind = L_ANISO_METAL; break;
    case RB_MAT_SDF_MATERIAL: m.kind = L_LAMBERTIAN; break;
    case RB_MAT_THIN_FILM: m.kind = L_THIN_FILM; break;
    case RB_MAT_CLEAR_COAT:
      m.kind = L_CLEAR_COAT;
      m.ior = d.refractive_index > 1.0f ? d.refractive_index : 1.5f;
      break;
    default: m.kind = L_ABSORB; break;
  }
  return m;
}

static void put(float4 *r, int w, float v) { reinterpret_cast<float *>(r)[w] = v; }
static float getw(const float4 *r, int w) { return reinterpret_cast<const float *>(r)[w]; }

// Rotation (radians, X then Y then Z) to a world->local matrix.
static void rot_matrix(const double r[3], float out[9]) {
  const double cx = std::cos(r[0]), sx = std::sin(r[0]);
  const double cy = std::cos(r[1]), sy = std::sin(r[1]);
  const double cz = std::cos(r[2]), sz = std::sin(r[2]);
  // local->world R = Rz * Ry * Rx; world->local = R^T
  const double R[3][3] = {
      {cz * cy, cz * sy * sx - sz * cx, cz * sy * cx + sz * sx},
      {sz * cy, sz * sy * sx + cz * cx, sz * sy * cx - cz * sx},
      {-sy, cy * sx, cy * cx}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[3 * i + j] = (float)R[j][i];
}

// Runs fn(begin, end) over [0, n) in contiguous chunks on the host's cores.
template <class F>
static void parallel_chunks(size_t n, F fn) {
  const size_t threads = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 64);
  if (n < 65536 || threads == 1) {
    fn((size_t)0, n);
    return;
  }
  const size_t chunk = (n + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (size_t t = 0; t < threads; ++t) {
    const size_t b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) pool.emplace_back(fn, b, e);
  }
  for (auto &th : pool) th.join();
}

static bool build_device_layout(const HostScene &hs, const rb_upload_opts &opts, HostLayout &L) {
  const size_t n = hs.geoms.size();
  L.prims.resize(3 * n);  // uninitialised: each record is zeroed by the thread that converts it
  L.mats.resize(hs.materials.size());
  for (size_t i = 0; i < hs.materials.size(); ++i) L.mats[i] = resolve_material(hs.materials[i]);
  // scene-wide flags in one parallel pass over the geometries
  std::atomic<bool> f_normals{false}, f_sdf{false}, f_displaced{false};
  parallel_chunks(n, [&](size_t b, size_t e) {
    bool nrm = false, sdf = false, disp = false;
    for (size_t i = b; i < e; ++i) {
      const Geom &g = hs.geoms[i];
      nrm |= (g.type == RB_GEOM_TRIANGLE && g.has_normals);
      sdf |= g.type == RB_GEOM_SDF_PRIMITIVE;
      disp |= g.type == RB_GEOM_DISPLACED_SPHERE;
    }
    if (nrm) f_normals.store(true, std::memory_order_relaxed);
    if (sdf) f_sdf.store(true, std::memory_order_relaxed);
    if (disp) f_displaced.store(true, std::memory_order_relaxed);
  });
  const bool any_normals = f_normals.load(), any_sdf = f_sdf.load(), any_displaced = f_displaced.load();
  bool any_light_mat = false;
  for (const auto &m : L.mats) any_light_mat |= m.kind == L_LIGHT;
  if (any_normals) L.normals.assign(3 * n, make_float4(0, 0, 0, 0));
  L.sdf.clear();
  double light_area = 0.0;
  auto tag_of = [&](const Geom &g, uint32_t kind) {
    const uint32_t mat =
        (g.material_id >= 0 && g.material_id < (int)hs.materials.size()) ? (uint32_t)g.material_id : 0xFFFFFFu;
    return kind | ((uint32_t)(g.visible ? 1 : 0) << 3) | ((uint32_t)((g.has_normals && any_normals) ? 1 : 0) << 4) |
           (mat << 8);
  };
  // records of spheres, quads and triangles, in parallel (each writes its own
  // slots); SDF primitives and emitters follow in order below
  parallel_chunks(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      const Geom &g = hs.geoms[i];
      float4 *r = &L.prims[3 * i];
      std::memset(r, 0, 3 * sizeof(float4));
      uint32_t kind = PK_NONE;
      switch (g.type) {
        case RB_GEOM_SPHERE:
        case RB_GEOM_DISPLACED_SPHERE:
          kind = g.type == RB_GEOM_SPHERE ? PK_SPHERE : PK_DISPLACED;
          for (int k = 0; k < 4; ++k) put(r, k, (float)g.p[k]);
          break;
        case RB_GEOM_RECTANGLE:
          kind = PK_RECT;
          for (int k = 0; k < 9; ++k) put(r, k, (float)g.p[k]);
          break;
        case RB_GEOM_TRIANGLE: {
          kind = PK_TRI;
          float v[9];
          for (int k = 0; k < 9; ++k) v[k] = (float)g.p[k];
          for (int k = 0; k < 3; ++k) {
            put(r, k, v[k]);
            put(r, 3 + k, ftz_sub(v[3 + k], v[k]));
            put(r, 6 + k, ftz_sub(v[6 + k], v[k]));
          }
          if (g.has_normals && any_normals)
            for (int k = 0; k < 3; ++k)
              L.normals[3 * i + k] =
                  make_float4((float)g.p[9 + 3 * k], (float)g.p[10 + 3 * k], (float)g.p[11 + 3 * k], 0.0f);
          break;
        }
        case RB_GEOM_SDF_PRIMITIVE:
          continue;  // below, in order (the SDF table index)
        default:
          kind = PK_NONE;  // CUBE / TRIANGLE_MESH are not converted (scene_builder_cuda.cu:138-140)
          break;
      }
      put(r, 11, __uint_as_float_host(tag_of(g, kind)));
    }
  });
  // SDF table and emitters, in geometry order; only scenes that hold either need the pass
  const size_t n_walk = (any_sdf || any_light_mat) ? n : 0;
  for (size_t i = 0; i < n_walk; ++i) {
    const Geom &g = hs.geoms[i];
    float4 *r = &L.prims[3 * i];
    uint32_t kind = tag_kind(__float_as_uint_host(getw(r, 11)));
    if (g.type == RB_GEOM_SDF_PRIMITIVE) {
      kind = PK_SDF;
      SdfPrim q;
      std::memset(&q, 0, sizeof q);
      const int t = (int)g.p[0];
      q.type = (t == RB_SDF_ROUND_BOX) ? 32 : t;
      q.material = g.material_id;
      q.px = (float)g.p[1]; q.py = (float)g.p[2]; q.pz = (float)g.p[3];
      q.a = (float)g.p[4]; q.b = (float)g.p[5]; q.c = (float)g.p[6];
      if (t != RB_SDF_SPHERE && t != RB_SDF_BOX && t != RB_SDF_ROUND_BOX && t != RB_SDF_TORUS &&
          t != RB_SDF_CAPSULE) {
        put(r, 11, __uint_as_float_host(tag_of(g, PK_NONE)));
        continue;
      }
      const double bound = sdf_bound_radius(g);
      // rounded box: half extents in params, rounding radius = 0.2 x the smallest half extent
      if (t == RB_SDF_ROUND_BOX) q.round = (float)(0.2 * std::min(g.p[4], std::min(g.p[5], g.p[6])));
      float R[9];
      const double rr[3] = {g.p[7], g.p[8], g.p[9]};
      rot_matrix(rr, R);
      q.r00 = R[0]; q.r01 = R[1]; q.r02 = R[2]; q.r10 = R[3]; q.r11 = R[4]; q.r12 = R[5];
      q.r20 = R[6]; q.r21 = R[7]; q.r22 = R[8];
      const double pad = hs.sdf.blend_k + 1e-3;
      put(r, 0, q.px); put(r, 1, q.py); put(r, 2, q.pz); put(r, 3, (float)(bound * 1.0001 + pad));
      put(r, 4, __int_as_float_host((int)L.sdf.size()));
      // convex primitives (their distance is convex along a ray) allow the field march's convex skip
      const bool convex = t == RB_SDF_SPHERE || t == RB_SDF_BOX || t == RB_SDF_ROUND_BOX || t == RB_SDF_CAPSULE;
      put(r, 5, __int_as_float_host(convex ? 1 : 0));
      q.bound_r = getw(r, 3);
      q.convex = convex ? 1 : 0;
      L.sdf.push_back(q);
      put(r, 11, __uint_as_float_host(tag_of(g, kind)));
    }
    // emitters for next-event estimation
    const uint32_t mat = (uint32_t)tag_material(__float_as_uint_host(getw(r, 11))) & 0xFFFFFFu;
    if (mat != 0xFFFFFFu && L.mats[mat].kind == L_LIGHT &&
        (kind == PK_RECT || kind == PK_TRI || kind == PK_SPHERE)) {
      const DevMaterial &m = L.mats[mat];
      if (m.emission.x > 0 || m.emission.y > 0 || m.emission.z > 0) {
        double area = 0.0;
        if (kind == PK_SPHERE) area = 4.0 * M_PI * (double)getw(r, 3) * (double)getw(r, 3);
        else {
          const double ax = getw(r, 3), ay = getw(r, 4), az = getw(r, 5);
          const double bx = getw(r, 6), by = getw(r, 7), bz = getw(r, 8);
          const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
          area = std::sqrt(cx * cx + cy * cy + cz * cz) * (kind == PK_TRI ? 0.5 : 1.0);
        }
        if (area > 0) {
          light_area += area;
          LightRec lr;
          lr.prim = (int)i;
          lr.area = (float)area;
          lr.cdf = (float)light_area;
          lr.pad = 0;
          L.lights.push_back(lr);
        }
      }
    }
  }
  L.light_area = (float)light_area;
  // smallest kernel class covering the scene (materials and primitive kinds)
  L.ms = RB_MS_DIFFUSE;
  for (const auto &m : L.mats) {
    if (m.kind == L_MIRROR || m.kind == L_ROUGH_MIRROR || m.kind == L_GLASS) L.ms = std::max(L.ms, RB_MS_CLASSIC);
    if (m.kind == L_ANISO_METAL || m.kind == L_THIN_FILM || m.kind == L_CLEAR_COAT || m.pattern) L.ms = RB_MS_FULL;
  }
  if (any_displaced) L.ms = std::max(L.ms, RB_MS_FULL);
  if (any_sdf) L.ms = RB_MS_SDF;
  if (!L.lights.empty()) L.lights.back().cdf = 3.0e38f;  // the last bin takes any rounding excess

  // BVH: interior nodes only, each holding its two children's boxes.
  L.use_bvh = hs.use_bvh && opts.use_bvh && !hs.nodes.empty() && hs.root >= 0;
  L.nodes.clear();
  L.root_ref = 0;
  for (int k = 0; k < 6; ++k) L.root_box[k] = 0.0f;
  if (L.use_bvh) {
    std::vector<int> remap(hs.nodes.size(), -1);
    int m = 0;
    for (size_t i = 0; i < hs.nodes.size(); ++i)
      if (!hs.nodes[i].is_leaf) remap[i] = m++;
    auto ref_of = [&](int i) -> int {
      const Node &c = hs.nodes[i];
      if (c.is_leaf) return make_leaf_ref(c.a, std::max(1, c.b));
      return remap[i];
    };
    for (const Node &nd : hs.nodes)
      if (nd.is_leaf && (nd.a >= (1 << 26) || nd.b > 32)) {
        set_error("BVH leaf beyond the device encoding");
        return false;
      }
    // interior node i goes to slot remap[i]: independent writes, in parallel
    L.nodes.resize(4 * (size_t)m);  // uninitialised: the loop below writes every word of every slot
    parallel_chunks(hs.nodes.size(), [&](size_t b, size_t e) {
      for (size_t i = b; i < e; ++i) {
        const Node &nd = hs.nodes[i];
        if (nd.is_leaf) continue;
        const Node &l = hs.nodes[nd.a], &rr = hs.nodes[nd.b];
        float4 *q = &L.nodes[4 * (size_t)remap[i]];
        float *w = reinterpret_cast<float *>(q);
        for (int k = 0; k < 3; ++k) { w[k] = (float)l.bmin[k]; w[3 + k] = (float)l.bmax[k]; }
        for (int k = 0; k < 3; ++k) { w[6 + k] = (float)rr.bmin[k]; w[9 + k] = (float)rr.bmax[k]; }
        int *wi = reinterpret_cast<int *>(&q[3]);
        wi[0] = ref_of(nd.a);
        wi[1] = ref_of(nd.b);
        wi[2] = nd.split_axis;
        wi[3] = 0;
      }
    });
    const Node &root = hs.nodes[hs.root];
    for (int k = 0; k < 3; ++k) { L.root_box[k] = (float)root.bmin[k]; L.root_box[3 + k] = (float)root.bmax[k]; }
    L.root_ref = ref_of(hs.root);
    if (opts.wide_bvh >= 0 && !opts.quantized_bvh) build_wide(L);  // 0: default on
    if (opts.quantized_bvh) {
      build_quantized(L);
      L.nodes.clear();  // the quantised copy replaces the FP32 nodes on the device
    }
  }
  L.groups.clear();
  if (opts.layout == RB_LAYOUT_GROUPS && hs.use_bvh && !hs.nodes.empty() && hs.root >= 0) {
    // the largest subtrees of at most G primitives, in leaf order; a subtree's
    // primitives are contiguous because the geometries are in the tree's leaf order
    const int G = std::max(1, opts.max_leaf);
    std::vector<int> first(hs.nodes.size()), count(hs.nodes.size());
    std::vector<std::pair<int, bool>> todo{{hs.root, false}};
    while (!todo.empty()) {  // post-order ranges
      const auto [ni, done] = todo.back();
      todo.pop_back();
      const Node &nd = hs.nodes[ni];
      if (nd.is_leaf) {
        first[ni] = nd.a;
        count[ni] = std::max(1, nd.b);
      } else if (done) {
        first[ni] = first[nd.a];
        count[ni] = count[nd.a] + count[nd.b];
      } else {
        todo.push_back({ni, true});
        todo.push_back({nd.b, false});
        todo.push_back({nd.a, false});
      }
    }
    std::vector<int> stack{hs.root};
    while (!stack.empty()) {  // pre-order, left child first: leaf order
      const int ni = stack.back();
      stack.pop_back();
      const Node &nd = hs.nodes[ni];
      if (nd.is_leaf || count[ni] <= G) {
        L.groups.push_back(make_float4((float)nd.bmin[0], (float)nd.bmin[1], (float)nd.bmin[2],
                                       __int_as_float_host(first[ni])));
        L.groups.push_back(make_float4((float)nd.bmax[0], (float)nd.bmax[1], (float)nd.bmax[2],
                                       __int_as_float_host(count[ni])));
      } else {
        stack.push_back(nd.b);
        stack.push_back(nd.a);
      }
    }
    L.use_bvh = false;
    L.nodes.clear();
    L.qnodes.clear();
    L.wnodes.clear();
  }
  return true;
}

// Host -> device copy of scene arrays. A copy from pageable memory goes
// through the driver's own small staging buffers at a few GB/s (471 MB of
// icosphere scene took about 0.13 s), so large arrays go through a pinned
// ring of four 32 MB buffers instead: the host cores fill one buffer while the
// copy engine drains the previous ones. The source is consumed before the
// call returns, as with a pageable cudaMemcpyAsync; a buffer is refilled only
// after the event of its last copy has completed.
namespace {
constexpr size_t kStageBytes = 32u << 20;
constexpr int kStages = 4;
struct UploadRing {
  std::mutex mu;
  char *buf[kStages] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t done[kStages] = {nullptr, nullptr, nullptr, nullptr};
  bool ready = false, failed = false;
};
UploadRing g_rings[64];  // one per device (events and buffers of that device's context)

// memcpy on up to eight host threads (more do not raise host memory bandwidth)
void copy_parallel(char *dst, const char *src, size_t n) {
  if (n < (1u << 20)) {  // below 1 MB a thread costs more than it copies
    std::memcpy(dst, src, n);
    return;
  }
  const size_t threads = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 8);
  const size_t chunk = (n + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (size_t t = 1; t < threads; ++t) {
    const size_t b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) pool.emplace_back([=] { std::memcpy(dst + b, src + b, e - b); });
  }
  std::memcpy(dst, src, std::min(n, chunk));
  for (auto &th : pool) th.join();
}
}  // namespace

static bool upload_bytes(void *dst, const void *src, size_t nb, cudaStream_t st) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (nb < 2 * kStageBytes || dev < 0 || dev >= 64)
    return cuda_ok(cudaMemcpyAsync(dst, src, nb, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(scene)");
  UploadRing &g_ring = g_rings[dev];
  std::lock_guard<std::mutex> lk(g_ring.mu);
  if (!g_ring.ready && !g_ring.failed) {
    bool ok = true;
    for (int k = 0; k < kStages && ok; ++k)
      ok = cudaMallocHost((void **)&g_ring.buf[k], kStageBytes) == cudaSuccess &&
           cudaEventCreateWithFlags(&g_ring.done[k], cudaEventDisableTiming) == cudaSuccess;
    if (ok) {
      g_ring.ready = true;
    } else {
      cudaGetLastError();  // not fatal: fall back to the pageable copy
      g_ring.failed = true;
    }
  }
  if (!g_ring.ready)
    return cuda_ok(cudaMemcpyAsync(dst, src, nb, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(scene)");
  const char *in = static_cast<const char *>(src);
  char *out = static_cast<char *>(dst);
  int k = 0;
  for (size_t off = 0; off < nb; off += kStageBytes, k = (k + 1) % kStages) {
    const size_t len = std::min(kStageBytes, nb - off);
    if (!cuda_ok(cudaEventSynchronize(g_ring.done[k]), "scene upload staging")) return false;
    char *stage = g_ring.buf[k];
    copy_parallel(stage, in + off, len);
    if (!cuda_ok(cudaMemcpyAsync(out + off, stage, len, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(scene)") ||
        !cuda_ok(cudaEventRecord(g_ring.done[k], st), "scene upload staging"))
      return false;
  }
  return true;
}

template <typename T, typename A>
static bool upload_vec(const std::vector<T, A> &v, T **dst, cudaStream_t st, size_t &bytes) {
  *dst = nullptr;
  if (v.empty()) return true;
  const size_t nb = v.size() * sizeof(T);
  if (!cuda_ok(cudaMalloc((void **)dst, nb), "cudaMalloc(scene)")) return false;
  bytes += nb;
  return upload_bytes(*dst, v.data(), nb, st);
}

void free_device_scene(DeviceScene *ds) {
  if (!ds) return;
  cudaFree((void *)ds->view.nodes);
  cudaFree((void *)ds->view.qnodes);
  cudaFree((void *)ds->view.wnodes);
  cudaFree((void *)ds->view.prims);
  cudaFree((void *)ds->view.normals);
  cudaFree((void *)ds->view.mats);
  cudaFree((void *)ds->view.lights);
  cudaFree((void *)ds->view.sdf);
  cudaFree((void *)ds->view.groups);
  cudaFree(ds->handle);
  delete ds;
}

DeviceScene *upload_scene(const HostScene &hs, const rb_upload_opts &opts, cudaStream_t st) {
  HostLayout L;
  if (!build_device_layout(hs, opts, L)) return nullptr;
  DeviceScene *ds = new DeviceScene();
  std::memset(&ds->view, 0, sizeof ds->view);
  SceneView &v = ds->view;
  size_t bytes = 0;
  float4 *nodes = nullptr, *prims = nullptr, *normals = nullptr;
  QNode *qn = nullptr;
  DevMaterial *mats = nullptr;
  LightRec *lights = nullptr;
  SdfPrim *sdf = nullptr;
  float4 *groups = nullptr;
  float4 *wn = nullptr;
  bool ok = upload_vec(L.nodes, &nodes, st, bytes) && upload_vec(L.qnodes, &qn, st, bytes) &&
            upload_vec(L.wnodes, &wn, st, bytes) &&
            upload_vec(L.prims, &prims, st, bytes) && upload_vec(L.normals, &normals, st, bytes) &&
            upload_vec(L.mats, &mats, st, bytes) && upload_vec(L.lights, &lights, st, bytes) &&
            upload_vec(L.sdf, &sdf, st, bytes) && upload_vec(L.groups, &groups, st, bytes);
  v.nodes = nodes; v.qnodes = qn; v.wnodes = wn; v.prims = prims; v.normals = normals; v.mats = mats;
  v.lights = lights; v.sdf = sdf; v.groups = groups;
  v.num_groups = (int)(L.groups.size() / 2);
  v.root_ref = L.root_ref;
  v.wide_root = L.wide_root;
  v.num_prims = (int)hs.geoms.size();
  v.num_mats = (int)hs.materials.size();
  v.num_lights = (int)L.lights.size();
  v.use_bvh = L.use_bvh ? 1 : 0;
  v.quantized = (L.use_bvh && opts.quantized_bvh) ? 1 : 0;
  v.num_sdf = (int)L.sdf.size();
  v.sdf_steps = hs.sdf.max_steps;
  v.sdf_eps = hs.sdf.epsilon;
  v.sdf_k = hs.sdf.blend_k;
  for (int k = 0; k < 6; ++k) v.root_box[k] = L.root_box[k];
  v.light_area = L.light_area;
  v.trav_budget = opts.traversal_budget > 0 ? opts.traversal_budget : 0;
  // The handle is a small device allocation so that it is a genuine device
  // pointer, as CudaScene::Scene* is in the reference (scene_builder_cuda.cu:294-296).
  // It holds a copy of the view and, in its last 8 bytes, the scene's
  // traversal-fault counter.
  static_assert(sizeof(SceneView) <= 248, "scene view must leave room for the fault counter");
  ok = ok && cuda_ok(cudaMalloc(&ds->handle, 256), "cudaMalloc(scene handle)") &&
       cuda_ok(cudaMemsetAsync(ds->handle, 0, 256, st), "cudaMemsetAsync(handle)");
  if (ok) v.faults = reinterpret_cast<unsigned long long *>(static_cast<char *>(ds->handle) + 248);
  ok = ok && cuda_ok(cudaMemcpyAsync(ds->handle, &v, sizeof v, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(handle)") &&
       cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize(upload)");
  ds->bytes = bytes + 256;
  ds->ms = L.ms;
  ds->layout_kind = !L.groups.empty() ? RB_LAYOUT_GROUPS : L.use_bvh ? RB_LAYOUT_LEAF : RB_LAYOUT_LINEAR;
  ds->layout_leaf = !L.groups.empty() ? std::max(1, opts.max_leaf) : L.use_bvh ? hs.max_leaf : 0;
  if (!ok) {
    free_device_scene(ds);
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  g_scenes[ds->handle] = ds;
  return ds;
}

void unregister_and_free(DeviceScene *ds) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_scenes.erase(ds->handle);
  }
  cudaDeviceSynchronize();
  free_device_scene(ds);
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
// Primary hits through pixel centres (offsets 0 in render_acc_kernel.cu:200-214).
__global__ void __launch_bounds__(256) k_primary(const RB_GRID_CONST SceneView S,
                                                    const RB_GRID_CONST FrameF P, int32_t *ids, float *tout) {
  extern __shared__ int2 smem[];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  if (x >= P.width || y >= P.height) return;
  Stack st;
  stack_init(st, smem, tid, blockDim.x * blockDim.y, S.short_stack);
  uint32_t ovf = 0;
  const f3 pc = P.p00 + ((float)x + 0.0f) * P.du + ((float)y + 0.0f) * P.dv;
  Ray r;
  r.o = P.center;
  r.d = pc - P.center;
  const HitInfo h = trace<false, RB_MS_SDF>(S, r, 0.001f, FLT_MAX, st, ovf);
  const int pix = y * P.width + x;
  ids[pix] = h.prim;
  if (tout) tout[pix] = h.prim >= 0 ? h.t : -1.0f;
}

// Adds the partial sums of sample slices 1..parts into the pixel sums, in
// slice order (Kahan-compensated when comp is given).
__global__ void k_fold_slices(float4 *__restrict__ acc, float4 *__restrict__ comp, const float4 *__restrict__ part,
                              int n, int parts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 a = acc[i];
  float4 c = comp ? comp[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  for (int z = 0; z < parts; ++z) {
    const float4 v = part[(size_t)z * n + i];
    if (comp) {
      kahan_add(a.x, c.x, v.x);
      kahan_add(a.y, c.y, v.y);
      kahan_add(a.z, c.z, v.z);
    } else {
      a.x += v.x; a.y += v.y; a.z += v.z;
    }
  }
  acc[i] = a;
  if (comp) comp[i] = c;
}

// accum float4 sums -> u8 (gammaCorrectKernel, render_acc_kernel.cu:11-44)
// (one thread per pixel on a 1-D grid: no grid.y limit on tall images)
__global__ void k_gamma(const float4 *__restrict__ acc, unsigned char *__restrict__ out, int npix, int spp, int ch,
                        float gamma, const int *__restrict__ counts) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npix) return;
  const float4 a = acc[pix];
  int n = counts ? abs(counts[pix]) : spp;
  if (n <= 0) n = 1;
  const float inv = 1.0f / (float)n, ig = 1.0f / gamma;
  const float r = fminf(powf(fmaxf(a.x * inv, 0.0f), ig), 0.999f);
  const float g = fminf(powf(fmaxf(a.y * inv, 0.0f), ig), 0.999f);
  const float b = fminf(powf(fmaxf(a.z * inv, 0.0f), ig), 0.999f);
  unsigned char *o = out + (size_t)pix * ch;
  o[0] = (unsigned char)(256.0f * r);
  o[1] = (unsigned char)(256.0f * g);
  o[2] = (unsigned char)(256.0f * b);
  if (ch == 4) o[3] = 255;
}

// Plasma colour ramp, 8 control points (the sample heat map's table,
// render_acc_kernel.cu:50-82).
__constant__ float c_plasma[8][4] = {
    {0.000f, 0.050f, 0.030f, 0.530f}, {0.143f, 0.230f, 0.015f, 0.660f}, {0.286f, 0.450f, 0.005f, 0.660f},
    {0.429f, 0.650f, 0.060f, 0.540f}, {0.571f, 0.820f, 0.170f, 0.360f}, {0.714f, 0.940f, 0.340f, 0.170f},
    {0.857f, 0.990f, 0.560f, 0.040f}, {1.000f, 0.940f, 0.975f, 0.130f}};

__global__ void k_heatmap(const int *__restrict__ counts, unsigned char *__restrict__ out, int npix, int ch,
                          int max_s) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npix) return;
  const int c = abs(counts[pix]);
  float t = max_s > 0 ? fminf((float)c / (float)max_s, 1.0f) : 0.0f;
  t = fminf(fmaxf(t, 0.0f), 1.0f);
  float r = c_plasma[7][1], g = c_plasma[7][2], b = c_plasma[7][3];
  for (int i = 0; i < 7; ++i) {
    if (t <= c_plasma[i + 1][0]) {
      const float lt = (t - c_plasma[i][0]) / (c_plasma[i + 1][0] - c_plasma[i][0]);
      r = c_plasma[i][1] + lt * (c_plasma[i + 1][1] - c_plasma[i][1]);
      g = c_plasma[i][2] + lt * (c_plasma[i + 1][2] - c_plasma[i][2]);
      b = c_plasma[i][3] + lt * (c_plasma[i + 1][3] - c_plasma[i][3]);
      break;
    }
  }
  unsigned char *o = out + (size_t)pix * ch;
  o[0] = (unsigned char)(255.0f * r);
  o[1] = (unsigned char)(255.0f * g);
  o[2] = (unsigned char)(255.0f * b);
  if (ch == 4) o[3] = 255;
}

__global__ void k_count_negative(const int *__restrict__ counts, int n, int *__restrict__ out) {
  int local = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) local += counts[i] < 0;
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, local);
}

__global__ void k_f3_to_f4(const float *__restrict__ in, float4 *__restrict__ out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_float4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.0f);
}
// float4 sums (minus their Kahan compensation terms when comp is given) to
// the host's float3 layout
__global__ void k_f4_to_f3(const float4 *__restrict__ in, const float4 *__restrict__ comp, float *__restrict__ out,
                           int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    float4 v = in[i];
    if (comp) {
      const float4 c = comp[i];
      v.x -= c.x;
      v.y -= c.y;
      v.z -= c.z;
    }
    out[3 * i] = v.x;
    out[3 * i + 1] = v.y;
    out[3 * i + 2] = v.z;
  }
}

// ---------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------
FrameF frame_from(const double *fr, int w, int h) {
  FrameF P;
  std::memset(&P, 0, sizeof P);
  auto g = [&](int i) { return f3((float)fr[3 * i], (float)fr[3 * i + 1], (float)fr[3 * i + 2]); };
  P.center = g(0);
  P.p00 = g(1);
  P.du = g(2);
  P.dv = g(3);
  P.cu = g(4);
  P.cv = g(5);
  P.width = w;
  P.height = h;
  return P;
}

int launch_primary(const DeviceScene *ds, const FrameF &P, int32_t *ids, float *t, cudaStream_t st) {
  dim3 blk(16, 16), grd((P.width + 15) / 16, (P.height + 15) / 16);
  const size_t sm = stack_smem_bytes(ds->view.short_stack, blk.x * blk.y);
  k_primary<<<grd, blk, sm, st>>>(ds->view, P, ids, t);
  g_launches++;
  return cuda_ok(cudaGetLastError(), "k_primary launch") ? RB_OK : RB_ERR_CUDA;
}

// Register budget (min resident blocks of 256 threads per SM) per material
// class; rb_render_opts.reserved[0] overrides it (the autotuner's knob).
// Defaults from a sweep on B200 (occupancy x block shape, per class).
static int default_minb(int ms, bool nee) {
  if (ms == RB_MS_DIFFUSE || ms == RB_MS_CLASSIC) return 4;
  if (ms == RB_MS_FULL) return nee ? 2 : 4;
  return 2;  // SDF
}
static void default_block(int ms, int &bx, int &by) {
  if (ms == RB_MS_CLASSIC) {
    bx = 16;
    by = 8;
    return;
  }
  bx = by = 8;  // 8x8 tiles: a warp's rays stay close together
}

// Stream-ordered scratch of the sample slices: a private memory pool per
// device that keeps its memory between calls (the default pool returns freed
// memory at every synchronisation, and mapping it again stalls the stream).
static cudaMemPool_t scratch_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {nullptr};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (!cuda_ok(cudaMemPoolCreate(&p, &props), "slice scratch pool")) return nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

static std::atomic<int> g_alloc_fail[RB_SITE_COUNT];

bool injected_alloc_failure(int site) {
  if (site < 0 || site >= RB_SITE_COUNT) return false;
  int n = g_alloc_fail[site].load();
  while (n > 0)
    if (g_alloc_fail[site].compare_exchange_weak(n, n - 1)) return true;
  return false;
}

// Opt-in per-kernel timing (rb_kernel_timer_enable): event pairs recorded on
// the launching stream around each k_render launch, read and released by
// rb_kernel_timer_read.
static std::atomic<bool> g_ktimer_on{false};
static std::mutex g_ktimer_mu;
static std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_ktimer_events;

static cudaEvent_t ktimer_mark(cudaStream_t st) {
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  cudaEventRecord(e, st);
  return e;
}

// Fetch mode's block size (two warps) and its resident blocks per SM per
// kernel instance (cached: the occupancy query is a driver call).
#define RB_FETCH_THREADS 64
// One k_render launch (launch == true) or its resident-block query, on the
// instances of the scene's node layout.
static int k_render_for(const DeviceScene *ds, bool launch, bool nee, int minb, dim3 grd, dim3 blk, size_t sm,
                        cudaStream_t st, const Globals &G, const FrameF &P, float4 *acc, float4 *comp, float4 *part,
                        int *counts, unsigned long long *counters, int *fetch, int nslices) {
  const SceneView &S = ds->view;
  if (S.use_bvh && S.wnodes)
    return k_render_dispatch_wide(launch, nee, ds->ms, minb, grd, blk, sm, st, S, G, P, acc, comp, part, counts,
                                  counters, fetch, nslices);
  return k_render_dispatch<RB_NODES_BINARY>(launch, nee, ds->ms, minb, grd, blk, sm, st, S, G, P, acc, comp, part,
                                            counts, counters, fetch, nslices);
}

static int fetch_resident_blocks(const DeviceScene *ds, bool nee, int minb, int sm) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  const int wide = ds->view.use_bvh && ds->view.wnodes ? 1 : 0;
  const auto key = std::make_tuple(dev, (ds->ms * 2 + (nee ? 1 : 0)) * 2 + wide, minb, sm, (int)RB_FETCH_THREADS);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  const int n = k_render_for(ds, false, nee, minb, dim3(1), dim3(RB_FETCH_THREADS), (size_t)sm, nullptr, Globals(),
                             FrameF(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0);
  std::lock_guard<std::mutex> lk(mu);
  cache[key] = n;
  return n;
}

int launch_render(const DeviceScene *ds, const Globals &G, const FrameF &P, float4 *acc, float4 *comp, int *counts,
                  unsigned long long *counters, cudaStream_t st) {
  const rb_render_opts o = current_opts();
  const int ms = ds->ms;
  int bx, by;
  default_block(ms, bx, by);
  if (ds->tuned_bx > 0 && ds->tuned_by > 0) {
    bx = ds->tuned_bx;
    by = ds->tuned_by;
  }
  // (whole warps: the kernel's warp shuffles take every lane)
  if (o.block_x > 0 && o.block_y > 0 && o.block_x * o.block_y <= 256 && o.block_x * o.block_y % 32 == 0) {
    bx = o.block_x;
    by = o.block_y;
  }
  // schedule: rb_render_opts.reserved[2] (1 grid, 2 fetch), else the scene's
  // tuned one, else fetch (measured on B200 against the grid at the same
  // register budget: icospheres 1920x1080 x 64 spp 33.6 -> 31.9 ms,
  // One-Weekend 400x225 x 32 spp 0.906 -> 0.869 ms, Cornell equal)
  const bool fetch_mode = o.reserved[2] > 0 ? o.reserved[2] == 2 : ds->tuned_fetch != 1;
  if (fetch_mode) {
    bx = RB_FETCH_THREADS;
    by = 1;
  }
  dim3 blk(bx, by), grd((P.width + bx - 1) / bx, (P.height + by - 1) / by);
  const size_t sm = stack_smem_bytes(ds->view.short_stack, blk.x * blk.y);
  // register budget: an explicit option, else the scene's tuned one (tuned
  // without next-event estimation, whose variant needs more registers), else
  // the class default
  const int minb = o.reserved[0] > 0 ? o.reserved[0]
                   : (ds->tuned_minb > 0 && !G.nee) ? ds->tuned_minb : default_minb(ms, G.nee != 0);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // A frame with fewer pixels than four times the GPU's resident threads
  // splits its samples into up to 8 slices (grid z in the grid schedule), so
  // that the launch keeps the GPU full to its end (measured on B200: 400x225 x
  // 32 spp 1.99 -> 1.13 ms, 512x512 x 256 spp 16.4 -> 15.1 ms); slices 1..
  // leave partial sums in a stream-ordered scratch buffer that k_fold_slices
  // adds in slice order. Splitting further (up to 16 times the resident
  // threads in pixel slices) ran slower on both (Cornell 512x512 x 51 spp
  // 3.35 -> 3.72 ms). Not with adaptive counts (their test needs each
  // pixel's whole batch in one thread).
  const long long npix = (long long)P.width * P.height;
  int slices = 1;
  if (!counts && P.samples > 1 && P.max_depth > 0) {
    if (o.reserved[1] > 0) {  // explicit slice count (rb_render_opts.reserved[1])
      slices = std::min(std::min(o.reserved[1], 64), P.samples);
    } else {
      const long long resident = (long long)sms * minb * 256;
      while (slices < 8 && slices * 2 <= P.samples && npix * slices < 4 * resident) slices *= 2;
    }
  }
  // one scratch allocation: the slices' partial sums, then fetch mode's work
  // counter (16-byte aligned after them)
  const size_t part_bytes = sizeof(float4) * (size_t)npix * (slices - 1);
  const size_t scratch_bytes = part_bytes + (fetch_mode ? 16 : 0);
  char *scratch = nullptr;
  if (scratch_bytes > 0) {
    cudaMemPool_t pool = scratch_pool();
    if (!pool || !cuda_ok(cudaMallocFromPoolAsync((void **)&scratch, scratch_bytes, pool, st), "launch scratch")) {
      if (fetch_mode) return RB_ERR_OUT_OF_MEMORY;
      slices = 1;  // the grid schedule renders without scratch
      scratch = nullptr;
    }
  }
  float4 *part = slices > 1 ? reinterpret_cast<float4 *>(scratch) : nullptr;
  int *fetch = nullptr;
  if (fetch_mode) {
    fetch = reinterpret_cast<int *>(scratch + part_bytes);
    cudaMemsetAsync(fetch, 0, sizeof(int), st);
    const long long items = (long long)((P.width + RB_TILE_W - 1) / RB_TILE_W) *
                            ((P.height + RB_TILE_H - 1) / RB_TILE_H) * slices;
    const long long per_sm = fetch_resident_blocks(ds, G.nee != 0, minb, (int)sm);
    const long long warps_per_block = RB_FETCH_THREADS / 32;
    grd = dim3((unsigned)std::max(1LL, std::min((long long)sms * per_sm, (items + warps_per_block - 1) / warps_per_block)),
               1, 1);
  } else {
    grd.z = slices;
  }
  cudaEvent_t t0 = g_ktimer_on.load(std::memory_order_relaxed) ? ktimer_mark(st) : nullptr;
  k_render_for(ds, true, G.nee != 0, minb, grd, blk, sm, st, G, P, acc, comp, part, counts, counters, fetch, slices);
  if (t0) {
    cudaEvent_t t1 = ktimer_mark(st);
    std::lock_guard<std::mutex> lk(g_ktimer_mu);
    if (t1) g_ktimer_events.emplace_back(t0, t1);
    else cudaEventDestroy(t0);
  }
  g_launches++;
  bool ok = cuda_ok(cudaGetLastError(), "k_render launch");
  if (part && ok) {
    k_fold_slices<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(acc, comp, part, (int)npix, slices - 1);
    g_launches++;
    ok = cuda_ok(cudaGetLastError(), "k_fold_slices launch");
  }
  if (scratch) cudaFreeAsync(scratch, st);
  return ok ? RB_OK : RB_ERR_CUDA;
}

// Display stream and pinned staging (renderer_cuda_device.cu:31-54).
static cudaStream_t s_display = nullptr;
static unsigned char *s_pinned = nullptr;
static size_t s_pinned_size = 0;
static unsigned char *s_dev_display = nullptr;
static size_t s_dev_display_size = 0;

static bool ensure_display(size_t bytes) {
  if (!s_dev_display || s_dev_display_size != bytes) {
    if (s_dev_display) cudaFree(s_dev_display);
    s_dev_display = nullptr;
    if (!cuda_ok(cudaMalloc(&s_dev_display, bytes), "cudaMalloc(display)")) return false;
    s_dev_display_size = bytes;
  }
  if (s_display && (!s_pinned || s_pinned_size != bytes)) {
    if (s_pinned) cudaFreeHost(s_pinned);
    s_pinned = nullptr;
    if (!cuda_ok(cudaMallocHost(&s_pinned, bytes), "cudaMallocHost(display)")) return false;
    s_pinned_size = bytes;
  }
  return true;
}

static void finish_display(unsigned char *out, size_t bytes) {
  if (s_display && s_pinned) {
    cudaMemcpyAsync(s_pinned, s_dev_display, bytes, cudaMemcpyDeviceToHost, s_display);
    cudaStreamSynchronize(s_display);
    std::memcpy(out, s_pinned, bytes);
  } else {
    cudaDeviceSynchronize();
    cudaMemcpy(out, s_dev_display, bytes, cudaMemcpyDeviceToHost);
  }
}

// ---------------------------------------------------------------------------
// Layout autotuner
// ---------------------------------------------------------------------------
// Candidate layouts are uploaded in turn and timed on a probe render of
// 256 x 256 pixels at 8 samples: the caller's camera subsampled to that size
// when given, otherwise two views of the scene's box (from its centre looking
// along +x, and from 1.5 box diagonals outside looking at the centre), so
// interior scenes and open scenes are both represented. The fastest
// candidate is kept.
static float probe_once(const DeviceScene *ds, const FrameF &P0, cudaStream_t st) {
  FrameF P = P0;
  const int W = P.width, H = P.height;
  float4 *acc = nullptr;
  if (!cuda_ok(cudaMallocAsync((void **)&acc, (size_t)W * H * 32, st), "autotune buffer")) return 1e30f;
  cudaMemsetAsync(acc, 0, (size_t)W * H * 32, st);
  Globals G = current_globals();
  G.nee = 0;
  G.dof_enabled = 0;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch_render(ds, G, P, acc, acc + W * H, nullptr, nullptr, st);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 3; ++r) {
    cudaEventRecord(a, st);
    launch_render(ds, G, P, acc, acc + W * H, nullptr, nullptr, st);
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFreeAsync(acc, st);
  cudaStreamSynchronize(st);
  return best;
}

static float probe_ms(const DeviceScene *ds, const std::vector<FrameF> &frames, cudaStream_t st);

// The scene's k_render launch configuration; the shared stack depth lives in
// the scene view, so the handle's device copy of the view is refreshed too.
static void apply_launch_choice(DeviceScene *ds, int minb, int bx, int by, int short_stack, cudaStream_t st) {
  ds->tuned_minb = minb;
  ds->tuned_bx = bx;
  ds->tuned_by = by;
  ds->view.short_stack = short_stack;
  cuda_ok(cudaMemcpyAsync(ds->handle, &ds->view, sizeof ds->view, cudaMemcpyHostToDevice, st), "tuned view");
  cudaStreamSynchronize(st);
}

// Second stage of the autotuner, on the chosen layout: the per-pixel kernel's
// register budget (2, 3 or 4 resident 256-thread blocks per SM) and block
// shape (8x8, 16x8, 16x16, 32x8), then, for BVH layouts, the traversal
// stack's shared-memory depth (4, 8, 16 entries). Each candidate is timed on
// the probe frames; the class defaults stay unless a candidate beats them by
// more than 2 %.
static void tune_launch(DeviceScene *ds, const std::vector<FrameF> &frames, cudaStream_t st) {
  int bx0, by0;
  default_block(ds->ms, bx0, by0);
  const int minb0 = default_minb(ds->ms, false);
  apply_launch_choice(ds, minb0, bx0, by0, RB_SHORT, st);
  float best = probe_ms(ds, frames, st);
  int bm = minb0, bbx = bx0, bby = by0, bsh = RB_SHORT;
  const int blocks[4][2] = {{8, 8}, {16, 8}, {16, 16}, {32, 8}};
  for (int m : {2, 3, 4})
    for (const auto &b : blocks) {
      if (m == minb0 && b[0] == bx0 && b[1] == by0) continue;
      apply_launch_choice(ds, m, b[0], b[1], RB_SHORT, st);
      const float t = probe_ms(ds, frames, st);
      if (t < 0.98f * best) {
        best = t;
        bm = m;
        bbx = b[0];
        bby = b[1];
      }
    }
  if (ds->layout_kind == RB_LAYOUT_LEAF && ds->view.use_bvh)
    for (int sh : {4, 16}) {
      apply_launch_choice(ds, bm, bbx, bby, sh, st);
      const float t = probe_ms(ds, frames, st);
      if (t < 0.98f * best) {
        best = t;
        bsh = sh;
      }
    }
  apply_launch_choice(ds, bm, bbx, bby, bsh, st);
  ds->probe_ms = best;
}

// Third stage, for scenes with a smooth SDF field (rendered by the wavefront
// engine): the engine's path slots (2, 4, 8 or 16 M), timed on a 16.8 M-path
// probe (the probe view at 256 samples per pixel; more paths than the largest
// candidate holds, so every candidate regenerates paths as in a real run).
static int tune_wavefront_queue(DeviceScene *ds, const FrameF &P0, cudaStream_t st) {
  const int W = P0.width, H = P0.height;
  double *acc = nullptr;
  if (!cuda_ok(cudaMalloc(&acc, sizeof(double) * 4 * (size_t)W * H), "wavefront probe buffer")) return 0;
  WfJob J;
  std::memset(&J, 0, sizeof J);
  J.P = P0;
  J.P.samples = 256;
  J.P.sample_base = 0;
  J.G = current_globals();
  J.G.nee = 0;
  J.G.dof_enabled = 0;
  J.acc = acc;
  int best_cap = 0;
  double best = 1e30;
  for (int cap : {1 << 21, 1 << 22, 1 << 23, 1 << 24}) {
    WfJob j = J;
    if (wf_render_jobs(ds, &j, 1, cap, nullptr, st) != RB_OK) break;  // also allocates at this capacity
    j = J;
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = wf_render_jobs(ds, &j, 1, cap, nullptr, st);
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != RB_OK) break;
    if (s < 0.98 * best) {
      best = s;
      best_cap = cap;
    }
  }
  cudaGetLastError();
  cudaFree(acc);
  return best_cap;
}

static std::vector<FrameF> probe_frames(const HostScene &hs, const rb_upload_opts &o, int depth) {
  std::vector<FrameF> out;
  const int W = 256, H = 256;
  auto finish = [&](FrameF P) {
    P.samples = 8;
    P.sample_base = 0;
    P.max_depth = depth;
    P.seed = 12345u;
    return P;
  };
  if (o.probe_frame && o.probe_width > 0 && o.probe_height > 0) {
    FrameF P = frame_from(o.probe_frame, W, H);
    const float sx = (float)o.probe_width / W, sy = (float)o.probe_height / H;
    P.du = P.du * sx;
    P.dv = P.dv * sy;
    out.push_back(finish(P));
    return out;
  }
  double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
  for (const Geom &g : hs.geoms) {
    lo[0] = std::min(lo[0], g.bmin.x); lo[1] = std::min(lo[1], g.bmin.y); lo[2] = std::min(lo[2], g.bmin.z);
    hi[0] = std::max(hi[0], g.bmax.x); hi[1] = std::max(hi[1], g.bmax.y); hi[2] = std::max(hi[2], g.bmax.z);
  }
  const V3 c((lo[0] + hi[0]) * 0.5, (lo[1] + hi[1]) * 0.5, (lo[2] + hi[2]) * 0.5);
  double diag = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                          (hi[2] - lo[2]) * (hi[2] - lo[2]));
  if (!(diag > 0) || diag > 1e6) diag = 10.0;
  double fr[21];
  camera_frame(c, c + V3(1.0, 0.0, 0.0), V3(0, 1, 0), 70.0, W, H, fr);
  out.push_back(finish(frame_from(fr, W, H)));
  camera_frame(c + (1.5 * diag) * unit(V3(1.0, 0.6, 1.3)), c, V3(0, 1, 0), 40.0, W, H, fr);
  out.push_back(finish(frame_from(fr, W, H)));
  return out;
}

static float probe_ms(const DeviceScene *ds, const std::vector<FrameF> &frames, cudaStream_t st) {
  float total = 0.f;
  for (const FrameF &P : frames) total += probe_once(ds, P, st);
  return total;
}

// Decisions are cached per (device, scene fingerprint): re-uploading the same
// scene (a renderer that rebuilds its device scene every frame) skips probing.
struct TuneKey {
  int dev;
  uint64_t fp;
  bool operator==(const TuneKey &o) const { return dev == o.dev && fp == o.fp; }
};
struct TuneKeyHash {
  size_t operator()(const TuneKey &k) const { return (size_t)(k.fp ^ ((uint64_t)k.dev << 56)); }
};
struct TuneChoice {
  bool linear;
  int leaf;    // BVH leaf size
  int groups;  // > 0: grouped linear layout with groups of at most this many primitives
  float probe_ms = 0.0f;  // the probe time that decided it
  int minb = 0, bx = 0, by = 0;  // k_render register budget and block shape
  int short_stack = 0;           // traversal stack entries in shared memory
  int wf_queue = 0;              // wavefront path slots (smooth-SDF scenes)
};
static std::unordered_map<TuneKey, TuneChoice, TuneKeyHash> g_tune_cache;

static uint64_t scene_fingerprint(const HostScene &hs) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
  mix(hs.geoms.size());
  mix(hs.materials.size());
  for (const Geom &g : hs.geoms) {
    uint64_t b[6];
    std::memcpy(&b[0], &g.bmin.x, 8); std::memcpy(&b[1], &g.bmin.y, 8); std::memcpy(&b[2], &g.bmin.z, 8);
    std::memcpy(&b[3], &g.bmax.x, 8); std::memcpy(&b[4], &g.bmax.y, 8); std::memcpy(&b[5], &g.bmax.z, 8);
    for (uint64_t v : b) mix(v);
    mix((uint64_t)g.type | ((uint64_t)(uint32_t)g.material_id << 8));
  }
  return h;
}

DeviceScene *autotune_upload(const HostScene &hs, const rb_upload_opts &o0, cudaStream_t st) {
  const int depth = o0.tune_depth > 0 ? o0.tune_depth : 8;
  const std::vector<FrameF> frames = probe_frames(hs, o0, depth);
  using Cand = TuneChoice;
  std::vector<Cand> cands;
  const size_t n = hs.geoms.size();
  int dev = 0;
  cudaGetDevice(&dev);
  const TuneKey key{dev, scene_fingerprint(hs)};
  bool cached = false;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      cands.push_back(it->second);
      cached = true;
    }
  }
  if (!cached) {
    if (n <= 4096) {
      cands.push_back({true, 0, 0});
      if (hs.use_bvh && !hs.nodes.empty())
        for (int G : {8, 16}) cands.push_back({false, 0, G});
    }
    if (n > 0) {
      // large scenes keep the tree they were built with (a rebuild costs seconds)
      // and tune only the launch configuration
      if (n > (1u << 20)) cands.push_back({false, hs.use_bvh && !hs.nodes.empty() ? hs.max_leaf : 4, 0});
      else for (int L : {1, 2, 4, 8}) cands.push_back({false, L, 0});
    }
  }
  DeviceScene *best = nullptr;
  float best_ms = 1e30f;
  for (const Cand &c : cands) {
    rb_upload_opts o = o0;
    o.layout = RB_LAYOUT_AS_BUILT;
    DeviceScene *ds = nullptr;
    if (c.linear) {
      o.use_bvh = 0;
      ds = upload_scene(hs, o, st);
    } else if (c.groups > 0) {
      o.use_bvh = 1;
      o.layout = RB_LAYOUT_GROUPS;
      o.max_leaf = c.groups;
      ds = upload_scene(hs, o, st);
    } else if (hs.use_bvh && hs.max_leaf == c.leaf && !hs.nodes.empty()) {
      o.use_bvh = 1;
      ds = upload_scene(hs, o, st);
    } else {
      HostScene copy = hs;
      copy.build_bvh(c.leaf, 0);
      o.use_bvh = 1;
      ds = upload_scene(copy, o, st);
    }
    if (!ds) continue;
    ds->layout_kind = c.linear ? RB_LAYOUT_LINEAR : c.groups > 0 ? RB_LAYOUT_GROUPS : RB_LAYOUT_LEAF;
    ds->layout_leaf = c.groups > 0 ? c.groups : c.leaf;
    if (cands.size() == 1) {  // cached (or only) choice: no probing
      ds->probe_ms = c.probe_ms;
      best = ds;
      break;
    }
    const float ms = probe_ms(ds, frames, st);
    ds->probe_ms = ms;
    if (ms < best_ms) {
      if (best) unregister_and_free(best);
      best = ds;
      best_ms = ms;
    } else {
      unregister_and_free(ds);
    }
  }
  if (!best) {
    set_error("rb_scene_upload: no layout could be uploaded");
    return nullptr;
  }
  if (cached) {
    const TuneChoice &c = cands[0];
    apply_launch_choice(best, c.minb, c.bx, c.by, c.short_stack, st);
    best->wf_queue = c.wf_queue;
    best->tune_cached = true;
    return best;
  }
  // The launch stage needs a probe that behaves like a full frame; for scenes
  // far larger than L2 (over 1 M primitives) a 256x256 probe does not (on the
  // 5.24 M-triangle scene its pick ran 9 % slower than the class defaults on
  // the full 1080p frame), so they keep the defaults.
  if (hs.geoms.size() <= (1u << 20)) tune_launch(best, frames, st);
  if (best->ms >= RB_MS_SDF && best->view.sdf_k > 0.0f && best->view.num_sdf > 0)
    best->wf_queue = tune_wavefront_queue(best, frames[0], st);
  {
    std::lock_guard<std::mutex> lk(g_mu);
    const bool groups = best->layout_kind == RB_LAYOUT_GROUPS;
    TuneChoice c{best->layout_kind == RB_LAYOUT_LINEAR, groups ? 0 : best->layout_leaf, groups ? best->layout_leaf : 0,
                 best->probe_ms};
    c.minb = best->tuned_minb;
    c.bx = best->tuned_bx;
    c.by = best->tuned_by;
    c.short_stack = best->view.short_stack;
    c.wf_queue = best->wf_queue;
    g_tune_cache[key] = c;
  }
  return best;
}

}  // namespace rb

// ===========================================================================
// C-ABI
// ===========================================================================
using namespace rb;

extern "C" {

void initCudaStreams(void) {
  if (!s_display) cuda_ok(cudaStreamCreateWithFlags(&s_display, cudaStreamNonBlocking), "initCudaStreams");
}

void cleanupCudaStreams(void) {
  if (s_display) {
    cudaStreamDestroy(s_display);
    s_display = nullptr;
  }
  if (s_pinned) {
    cudaFreeHost(s_pinned);
    s_pinned = nullptr;
    s_pinned_size = 0;
  }
}

void setLightIntensity(float v) { g_globals.light_intensity = v; }
void setBackgroundIntensity(float v) { g_globals.background_intensity = v; }
void setMetalFuzziness(float v) { g_globals.metal_fuzziness = v; }
void setGlassRefractionIndex(float v) { g_globals.glass_ior = v; }
void setDOFEnabled(bool e) { g_globals.dof_enabled = e ? 1 : 0; }
void setDOFAperture(float v) { g_globals.dof_aperture = v; }
void setDOFFocusDistance(float v) { g_globals.dof_focus = v; }

void rb_get_render_opts(rb_render_opts *o) {
  if (o) *o = g_opts;
}
void rb_set_render_opts(const rb_render_opts *o) {
  if (o) g_opts = *o;
}

// Buffers this library handed out came from its memory pool and go back to it
// in stream order (legacy default stream, as the reference's cudaFree is
// ordered after all prior work); anything else is released with cudaFree.
void freeDeviceRandomStates(void *p) {
  if (!p) return;
  bool ours = false;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    ours = g_rng_ctx.erase(p) > 0;
  }
  if (ours) cudaFreeAsync(p, 0);
  else cudaFree(p);
}

void freeDeviceAccumBuffer(void *p) {
  if (!p) return;
  bool ours = false;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    ours = g_accum_bytes.erase(p) > 0;
  }
  if (ours) cudaFreeAsync(p, 0);
  else cudaFree(p);
}

void resetDeviceAccumBuffer(void *p, int num_pixels) {
  if (!p || num_pixels <= 0) return;
  size_t bytes = (size_t)num_pixels * sizeof(float4);
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_accum_bytes.find(p);
    if (it != g_accum_bytes.end()) bytes = std::min(it->second, 2 * bytes);  // sums and compensation
  }
  cuda_ok(cudaMemset(p, 0, bytes), "resetDeviceAccumBuffer");
}

}  // extern "C"

namespace rb {
namespace {
// float3 staging of the drop-in's host accumulation buffer, kept per device
// across calls (the reference converts through a host loop; here a kernel
// converts on the device and one pinned copy crosses PCIe): a device float3
// array and a pinned host mirror, grown on demand, freed at exit.
struct F3Stage {
  float *dev = nullptr, *host = nullptr;
  size_t bytes = 0;
};
F3Stage g_f3_stage[64];
std::mutex g_stage_mu;

F3Stage *f3_stage(size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return nullptr;
  F3Stage &S = g_f3_stage[dev];
  if (S.bytes < bytes) {
    if (S.dev) cudaFree(S.dev);
    if (S.host) cudaFreeHost(S.host);
    S.dev = S.host = nullptr;
    S.bytes = 0;
    if (!cuda_ok(cudaMalloc(&S.dev, bytes), "cudaMalloc(accum staging)") ||
        !cuda_ok(cudaMallocHost(&S.host, bytes), "cudaMallocHost(accum staging)"))
      return nullptr;
    S.bytes = bytes;
  }
  return &S;
}
}  // namespace
}  // namespace rb

extern "C" {

unsigned long long renderPixelsCUDAAccumulative(
    unsigned char *image, float *accum_buffer, rb_cuda_scene *scene, int width, int height, double ccx,
    double ccy, double ccz, double p0x, double p0y, double p0z, double dux, double duy, double duz, double dvx,
    double dvy, double dvz, int samples_to_add, int total_samples_so_far, int max_depth, void **d_rand_states_ptr,
    void **d_accum_buffer_ptr, double cux, double cuy, double cuz, double cvx, double cvy, double cvz,
    void *d_pixel_sample_counts, int min_adaptive_samples, float adaptive_threshold) {
  (void)image;
  (void)total_samples_so_far;
  if (!scene) return 0ull;
  DeviceScene *ds = lookup_scene(scene);
  if (!ds) {
    set_error("renderPixelsCUDAAccumulative: scene handle was not created by this library");
    return 0ull;
  }
  if (width <= 0 || height <= 0 || samples_to_add < 0 || !d_rand_states_ptr || !d_accum_buffer_ptr) {
    set_error("renderPixelsCUDAAccumulative: invalid argument");
    return 0ull;
  }
  const int n = width * height;
  cudaStream_t st = 0;
  // RNG context: the per-path streams are counter based; the context keeps
  // the index of the next sample so that successive calls draw new samples.
  // Both allocations come from the per-device pool that keeps its memory, so a
  // renderer that allocates and frees them for every frame (RendererCUDA::render)
  // pays neither cudaMalloc nor the device-wide synchronisation of cudaFree
  // (measured: 2.4 ms more on a frame's first call, frees of 0.4 to 19 ms).
  cudaMemPool_t pool = scratch_pool();
  if (!pool) return 0ull;
  if (*d_rand_states_ptr == nullptr) {
    void *p = nullptr;
    if (!cuda_ok(cudaMallocFromPoolAsync(&p, 256, pool, st), "rng context")) return 0ull;
    *d_rand_states_ptr = p;
    std::lock_guard<std::mutex> lk(g_mu);
    g_rng_ctx[p] = 0;
  }
  float4 *acc = nullptr;
  const size_t nb = (size_t)n * sizeof(float4);
  if (*d_accum_buffer_ptr == nullptr) {
    if (!cuda_ok(cudaMallocFromPoolAsync((void **)&acc, 2 * nb, pool, st), "accumulation buffer")) return 0ull;
    *d_accum_buffer_ptr = acc;
    {
      std::lock_guard<std::mutex> lk(g_mu);
      g_accum_bytes[acc] = 2 * nb;
    }
    cudaMemsetAsync(acc, 0, 2 * nb, st);
    if (accum_buffer) {
      std::lock_guard<std::mutex> lk(g_stage_mu);
      F3Stage *S = f3_stage((size_t)n * 12);
      if (!S) return 0ull;
      std::memcpy(S->host, accum_buffer, (size_t)n * 12);
      cudaMemcpyAsync(S->dev, S->host, (size_t)n * 12, cudaMemcpyHostToDevice, st);
      k_f3_to_f4<<<(n + 255) / 256, 256, 0, st>>>(S->dev, acc, n);
      g_launches++;
      if (!cuda_ok(cudaStreamSynchronize(st), "accum upload")) return 0ull;
    }
  } else {
    acc = static_cast<float4 *>(*d_accum_buffer_ptr);
  }
  float4 *comp = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_accum_bytes.find(acc);
    if (it != g_accum_bytes.end() && it->second >= 2 * nb) comp = acc + n;
  }
  uint32_t base = 0;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_rng_ctx.find(*d_rand_states_ptr);
    if (it != g_rng_ctx.end()) {
      base = it->second;
      it->second += (uint32_t)samples_to_add;
    }
  }
  const double fr[21] = {ccx, ccy, ccz, p0x, p0y, p0z, dux, duy, duz, dvx, dvy, dvz, cux, cuy, cuz, cvx, cvy, cvz, 0, 0, 0};
  FrameF P = frame_from(fr, width, height);
  P.samples = samples_to_add;
  P.sample_base = (int)base;
  P.max_depth = max_depth;
  P.seed = current_opts().seed;
  P.salt = 0;
  P.min_adaptive = min_adaptive_samples;
  P.adaptive_threshold = adaptive_threshold;
  const rb_render_opts o = current_opts();
  if (samples_to_add > 0)
    launch_render(ds, current_globals(), P, acc, o.kahan ? comp : nullptr, static_cast<int *>(d_pixel_sample_counts),
                  nullptr, st);
  cuda_ok(cudaStreamSynchronize(st), "renderPixelsCUDAAccumulative");
  if (accum_buffer) {
    std::lock_guard<std::mutex> lk(g_stage_mu);
    F3Stage *S = f3_stage((size_t)n * 12);
    if (S) {
      k_f4_to_f3<<<(n + 255) / 256, 256, 0, st>>>(acc, comp, S->dev, n);
      g_launches++;
      cudaMemcpyAsync(S->host, S->dev, (size_t)n * 12, cudaMemcpyDeviceToHost, st);
      if (cuda_ok(cudaStreamSynchronize(st), "accum download")) std::memcpy(accum_buffer, S->host, (size_t)n * 12);
    }
  }
  return (unsigned long long)n * (unsigned long long)samples_to_add;
}

void convertAccumToDisplayCUDA(void *d_acc, unsigned char *img, int w, int h, int ch, int spp, float gamma,
                               void *counts) {
  if (!d_acc || !img || spp <= 0 || w <= 0 || h <= 0 || (int64_t)w * h > INT32_MAX) return;
  const size_t bytes = (size_t)w * h * ch;
  if (!ensure_display(bytes)) return;
  const int npix = w * h;
  cudaStream_t st = s_display ? s_display : 0;
  k_gamma<<<(npix + 255) / 256, 256, 0, st>>>(static_cast<const float4 *>(d_acc), s_dev_display, npix, spp, ch, gamma,
                                               static_cast<const int *>(counts));
  g_launches++;
  finish_display(img, bytes);
}

void allocateAdaptiveBuffer(void **p, int n) {
  if (!p || *p) return;
  if (cuda_ok(cudaMalloc(p, (size_t)n * sizeof(int)), "allocateAdaptiveBuffer"))
    cudaMemset(*p, 0, (size_t)n * sizeof(int));
}
void resetAdaptiveBuffer(void *p, int n) {
  if (p) cudaMemset(p, 0, (size_t)n * sizeof(int));
}
void freeAdaptiveBuffer(void *p) {
  if (p) cudaFree(p);
}

int countConvergedPixels(void *p, int n) {
  if (!p || n <= 0) return 0;
  int *d = nullptr;
  if (!cuda_ok(cudaMalloc(&d, sizeof(int)), "countConvergedPixels")) return 0;
  cudaMemset(d, 0, sizeof(int));
  k_count_negative<<<std::min(1184, (n + 255) / 256), 256>>>(static_cast<const int *>(p), n, d);
  g_launches++;
  int out = 0;
  cudaMemcpy(&out, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return out;
}

void renderSampleHeatmapCUDA(void *counts, unsigned char *img, int w, int h, int ch, int max_s) {
  if (!counts || !img || w <= 0 || h <= 0 || (int64_t)w * h > INT32_MAX) return;
  const size_t bytes = (size_t)w * h * ch;
  if (!ensure_display(bytes)) return;
  const int npix = w * h;
  k_heatmap<<<(npix + 255) / 256, 256, 0, s_display ? s_display : 0>>>(static_cast<const int *>(counts), s_dev_display,
                                                                       npix, ch, max_s);
  g_launches++;
  finish_display(img, bytes);
}

rb_cuda_scene *rb_scene_upload(const rb_scene_desc *s, const rb_upload_opts *opts, void *stream) {
  if (!s) {
    set_error("rb_scene_upload: null scene");
    return nullptr;
  }
  rb_upload_opts o;
  std::memset(&o, 0, sizeof o);
  o.use_bvh = 1;
  if (opts) o = *opts;
  const HostScene &hs = host_scene_of(s);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DeviceScene *ds = nullptr;
  try {
    if (o.layout == RB_LAYOUT_AUTOTUNE) {
      ds = autotune_upload(hs, o, st);
    } else if (o.layout == RB_LAYOUT_LINEAR) {
      o.use_bvh = 0;
      ds = upload_scene(hs, o, st);
      if (ds) ds->layout_kind = RB_LAYOUT_LINEAR;
    } else if (o.layout == RB_LAYOUT_LEAF && o.max_leaf >= 1 && o.max_leaf <= 32 && o.max_leaf != hs.max_leaf) {
      HostScene copy = hs;
      copy.build_bvh(o.max_leaf, 0);
      ds = upload_scene(copy, o, st);
    } else {
      ds = upload_scene(hs, o, st);
    }
  } catch (const std::exception &e) {
    set_error(std::string("rb_scene_upload: ") + e.what());
    return nullptr;
  }
  return ds ? static_cast<rb_cuda_scene *>(ds->handle) : nullptr;
}

int rb_scene_tuning(const rb_cuda_scene *scene, rb_tuning *out) {
  DeviceScene *ds = lookup_scene(scene);
  if (!ds) return RB_ERR_NOT_FOUND;
  if (!out) return RB_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof *out);
  out->layout = ds->layout_kind;
  out->leaf = ds->layout_leaf;
  out->blocks_per_sm = ds->tuned_minb;
  out->block_x = ds->tuned_bx;
  out->block_y = ds->tuned_by;
  out->short_stack = ds->view.short_stack;
  out->wavefront_queue = ds->wf_queue;
  out->probe_ms = ds->probe_ms;
  out->from_cache = ds->tune_cached ? 1 : 0;
  return RB_OK;
}

int rb_scene_layout_info(const rb_cuda_scene *scene, int *kind, int *leaf, float *probe_ms) {
  DeviceScene *ds = lookup_scene(scene);
  if (!ds) return RB_ERR_NOT_FOUND;
  if (kind) *kind = ds->layout_kind;
  if (leaf) *leaf = ds->layout_leaf;
  if (probe_ms) *probe_ms = ds->probe_ms;
  return RB_OK;
}

void rb_scene_free_device(rb_cuda_scene *scene) {
  if (!scene) return;
  DeviceScene *ds = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_scenes.find(scene);
    if (it == g_scenes.end()) return;
    ds = it->second;
    g_scenes.erase(it);
  }
  cudaDeviceSynchronize();
  free_device_scene(ds);
}

int rb_scene_traversal_faults(const rb_cuda_scene *scene, uint64_t *count, int reset) {
  DeviceScene *ds = lookup_scene(scene);
  if (!ds) {
    set_error("rb_scene_traversal_faults: unknown scene handle");
    return RB_ERR_NOT_FOUND;
  }
  unsigned long long n = 0;
  if (!cuda_ok(cudaDeviceSynchronize(), "rb_scene_traversal_faults") ||
      !cuda_ok(cudaMemcpy(&n, ds->view.faults, sizeof n, cudaMemcpyDeviceToHost), "rb_scene_traversal_faults"))
    return RB_ERR_CUDA;
  if (reset && !cuda_ok(cudaMemset(ds->view.faults, 0, sizeof n), "rb_scene_traversal_faults")) return RB_ERR_CUDA;
  if (count) *count = n;
  return RB_OK;
}

int rb_scene_check_wide(const rb_scene_desc *s, int64_t out[4]) {
  if (!s || !out) {
    set_error("rb_scene_check_wide: null argument");
    return RB_ERR_INVALID_ARG;
  }
  const HostScene &hs = host_scene_of(s);
  rb_upload_opts o;
  std::memset(&o, 0, sizeof o);
  o.use_bvh = 1;
  HostLayout L;
  try {
    if (!build_device_layout(hs, o, L)) return RB_ERR_INVALID_ARG;
  } catch (const std::exception &e) {
    set_error(std::string("rb_scene_check_wide: ") + e.what());
    return RB_ERR_INVALID_ARG;
  }
  for (int k = 0; k < 4; ++k) out[k] = 0;
  if (!L.use_bvh) return RB_OK;
  // the binary tree's leaves, by first primitive
  std::unordered_map<int, int> leaves;  // first -> times reached in the wide tree
  const size_t nbin = L.nodes.size() / 4;
  auto note_leaf = [&](int r) { leaves.emplace(leaf_first(r), 0); };
  if (ref_is_leaf(L.root_ref)) note_leaf(L.root_ref);
  for (size_t i = 0; i < nbin; ++i) {
    const int *wi = reinterpret_cast<const int *>(&L.nodes[4 * i + 3]);
    for (int c = 0; c < 2; ++c)
      if (ref_is_leaf(wi[c])) note_leaf(wi[c]);
  }
  out[2] = (int64_t)leaves.size();
  const int64_t nwide = (int64_t)(L.wnodes.size() / 8);
  out[0] = nwide;
  if (nwide == 0) {  // a leaf root keeps the binary root
    out[1] = ref_is_leaf(L.wide_root) ? 1 : 0;
    return out[1] == out[2] ? RB_OK : RB_ERR_INVALID_ARG;
  }
  std::vector<std::pair<int, int>> todo{{L.wide_root, 1}};
  std::vector<char> seen(nwide, 0);
  int64_t reached = 0;
  while (!todo.empty()) {
    const auto [n, depth] = todo.back();
    todo.pop_back();
    if (n < 0 || n >= nwide || seen[n]) {
      set_error("rb_scene_check_wide: wide node out of range or reached twice");
      return RB_ERR_INVALID_ARG;
    }
    seen[n] = 1;
    out[3] = std::max<int64_t>(out[3], depth);
    const float *w = reinterpret_cast<const float *>(&L.wnodes[8 * (size_t)n]);
    const int *r = reinterpret_cast<const int *>(&L.wnodes[8 * (size_t)n + 6]);
    for (int c = 0; c < 4; ++c) {
      if (!std::isfinite(w[c])) continue;  // empty slot
      if (ref_is_leaf(r[c])) {
        auto it = leaves.find(leaf_first(r[c]));
        if (it == leaves.end() || it->second++ > 0) {
          set_error("rb_scene_check_wide: a leaf missing from the binary tree or reached twice");
          return RB_ERR_INVALID_ARG;
        }
        ++reached;
        continue;
      }
      if (r[c] < 0 || r[c] >= nwide) {
        set_error("rb_scene_check_wide: child ref out of range");
        return RB_ERR_INVALID_ARG;
      }
      // the child's slot box bounds every box inside the child node
      const float *cw = reinterpret_cast<const float *>(&L.wnodes[8 * (size_t)r[c]]);
      for (int g = 0; g < 4; ++g) {
        if (!std::isfinite(cw[g])) continue;
        for (int k = 0; k < 3; ++k)
          if (cw[8 * k + g] < w[8 * k + c] || cw[8 * k + 4 + g] > w[8 * k + 4 + c]) {
            set_error("rb_scene_check_wide: a child box outside its slot box");
            return RB_ERR_INVALID_ARG;
          }
      }
      todo.push_back({r[c], depth + 1});
    }
  }
  out[1] = reached;
  for (int64_t i = 0; i < nwide; ++i)
    if (!seen[i]) {
      set_error("rb_scene_check_wide: unreachable wide node");
      return RB_ERR_INVALID_ARG;
    }
  return reached == out[2] ? RB_OK : RB_ERR_INVALID_ARG;
}

int64_t rb_scene_device_bytes(const rb_cuda_scene *scene) {
  DeviceScene *ds = lookup_scene(scene);
  return ds ? (int64_t)ds->bytes : 0;
}

int rb_primary_hits(const rb_cuda_scene *scene, int w, int h, const double frame[21], int32_t *ids, float *t,
                    void *stream) {
  DeviceScene *ds = lookup_scene(scene);
  if (!ds) {
    set_error("rb_primary_hits: unknown scene handle");
    return RB_ERR_NOT_FOUND;
  }
  if (w <= 0 || h <= 0 || !frame || !ids) {
    set_error("rb_primary_hits: invalid argument");
    return RB_ERR_INVALID_ARG;
  }
  return launch_primary(ds, frame_from(frame, w, h), ids, t, static_cast<cudaStream_t>(stream));
}

int rb_render_accumulate(const rb_cuda_scene *scene, int w, int h, const double frame[21], int samples,
                         int sample_base, int max_depth, float *accum, float *comp, uint64_t *counters,
                         void *stream) {
  DeviceScene *ds = lookup_scene(scene);
  if (!ds) {
    set_error("rb_render_accumulate: unknown scene handle");
    return RB_ERR_NOT_FOUND;
  }
  if (w <= 0 || h <= 0 || !frame || !accum || samples < 0 || max_depth < 0 || sample_base < 0) {
    set_error("rb_render_accumulate: invalid argument");
    return RB_ERR_INVALID_ARG;
  }
  if (samples == 0) return RB_OK;
  FrameF P = frame_from(frame, w, h);
  P.samples = samples;
  P.sample_base = sample_base;
  P.max_depth = max_depth;
  P.seed = current_opts().seed;
  P.salt = 0;
  return launch_render(ds, current_globals(), P, reinterpret_cast<float4 *>(accum), reinterpret_cast<float4 *>(comp),
                       nullptr, reinterpret_cast<unsigned long long *>(counters), static_cast<cudaStream_t>(stream));
}

unsigned long long rb_launch_count(void) { return g_launches.load(); }

void rb_kernel_timer_enable(int on) { g_ktimer_on.store(on != 0); }

int rb_inject_alloc_failures(const char *site, int count) {
  if (!site || count < 0) return RB_ERR_INVALID_ARG;
  const std::string s(site);
  const int k = s == "server_job" ? RB_SITE_SERVER_JOB : s == "wavefront_queue" ? RB_SITE_WAVEFRONT : -1;
  if (k < 0) {
    set_error("rb_inject_alloc_failures: unknown site (server_job, wavefront_queue)");
    return RB_ERR_INVALID_ARG;
  }
  g_alloc_fail[k].store(count);
  return RB_OK;
}

int rb_kernel_timer_read(double *ms, int64_t *launches) {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  {
    std::lock_guard<std::mutex> lk(g_ktimer_mu);
    ev.swap(g_ktimer_events);
  }
  double total = 0.0;
  int rc = RB_OK;
  for (auto &p : ev) {
    float m = 0.f;
    if (cuda_ok(cudaEventSynchronize(p.second), "rb_kernel_timer_read") &&
        cuda_ok(cudaEventElapsedTime(&m, p.first, p.second), "rb_kernel_timer_read"))
      total += m;
    else
      rc = RB_ERR_CUDA;
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
  if (ms) *ms = total;
  if (launches) *launches = (int64_t)ev.size();
  return rc;
}

}  // extern "C"
