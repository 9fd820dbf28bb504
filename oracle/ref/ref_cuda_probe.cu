// Oracle infrastructure (test-only): drives the reference's OWN CUDA render
// path, compiled from its unmodified .cu sources (oracle/ref/Makefile), on the
// GPU:
//   * scenes are built with the reference's SceneDescription / buildBVH and
//     uploaded with its Scene::CudaSceneBuilder::buildGPUScene
//     (gpu_renderers/scene_builder_cuda.cu:148-303);
//   * primary-hit ids: hit_scene (gpu_renderers/cuda_raytracer.cuh:487-602)
//     does not return the index of the primitive it hit, so the probe kernel
//     walks the same node stack calling the reference's own hit_aabb and
//     intersect_geometry and records that index; each ray is also run through
//     hit_scene itself and the probe reports any ray where the two disagree on
//     hit / distance (expected: none);
//   * images and timings come from the reference's renderPixelsCUDAAccumulative
//     (gpu_renderers/renderer_cuda_device.cu:157-322) called as its offline
//     renderer does (renderer_cuda_host.hpp:35-58).
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "cuda_raytracer.cuh"
#include "cuda_scene.cuh"
#include "renderer_cuda_device.cuh"
#include "scene_description.hpp"

namespace Scene {
class CudaSceneBuilder {
 public:
  static CudaScene::Scene *buildGPUScene(const SceneDescription &desc);
  static void freeGPUScene(CudaScene::Scene *scene);
};
}  // namespace Scene

struct RefGpuScene {
  Scene::SceneDescription *desc;
  CudaScene::Scene *dev;
};

__device__ int probe_closest(const CudaScene::Scene &scene, const ray_simple &r, float t_min, float t_max,
                             float &t_out) {
  hit_record_simple temp;
  float closest = t_max;
  int idx = -1;
  if (scene.use_bvh && scene.bvh_root_idx >= 0) {
    int stack[32];
    int sp = 0;
    stack[sp++] = scene.bvh_root_idx;
    while (sp > 0) {
      const int ni = stack[--sp];
      const CudaScene::BVHNode &node = scene.bvh_nodes[ni];
      if (!hit_aabb(r, node.bounds_min, node.bounds_max, t_min, closest)) continue;
      if (node.is_leaf) {
        const int first = node.data.leaf.first_geom_idx, count = node.data.leaf.geom_count;
        for (int i = 0; i < count; ++i) {
          if (intersect_geometry(scene.geometries[first + i], r, t_min, closest, temp)) {
            closest = temp.t;
            idx = first + i;
          }
        }
      } else {
        const float dc = node.split_axis == 0 ? r.dir.x : (node.split_axis == 1 ? r.dir.y : r.dir.z);
        const int nearc = dc >= 0.0f ? node.data.interior.left_child : node.data.interior.right_child;
        const int farc = dc >= 0.0f ? node.data.interior.right_child : node.data.interior.left_child;
        if (sp < 32) stack[sp++] = farc;
        if (sp < 32) stack[sp++] = nearc;
      }
    }
  } else {
    for (int i = 0; i < scene.num_geometries; ++i) {
      if (intersect_geometry(scene.geometries[i], r, t_min, closest, temp)) {
        closest = temp.t;
        idx = i;
      }
    }
  }
  t_out = closest;
  return idx;
}

__global__ void probe_kernel(const CudaScene::Scene *__restrict__ scene, int w, int h, float ccx, float ccy, float ccz,
                             float p0x, float p0y, float p0z, float dux, float duy, float duz, float dvx, float dvy,
                             float dvz, int *ids, float *ts, int *disagree) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  f3 camera_center(ccx, ccy, ccz), pixel00_loc(p0x, p0y, p0z), pixel_delta_u(dux, duy, duz), pixel_delta_v(dvx, dvy, dvz);
  const float offset_u = 0.0f, offset_v = 0.0f;
  f3 pixel_center = pixel00_loc + ((float)x + offset_u) * pixel_delta_u + ((float)y + offset_v) * pixel_delta_v;
  f3 ray_direction = pixel_center - camera_center;
  ray_simple r(camera_center, ray_direction);
  float t;
  const int idx = probe_closest(*scene, r, 0.001f, FLT_MAX, t);
  hit_record_simple rec;
  const bool hit = hit_scene(*scene, r, 0.001f, FLT_MAX, rec);
  if (hit != (idx >= 0) || (hit && rec.t != t)) atomicAdd(disagree, 1);
  ids[y * w + x] = idx;
  ts[y * w + x] = idx >= 0 ? t : -1.0f;
}

extern "C" {

void *refc_scene_create(const void *materials, int nmat, int mat_size, const uint8_t *kinds, const double *params,
                        const int32_t *mats, int64_t n, int build_bvh);
void refc_scene_destroy(void *s);

int refc_primary(void *sp, int w, int h, const double *fr, int *ids_host, float *t_host) {
  auto *s = static_cast<RefGpuScene *>(sp);
  int *d_ids = nullptr, *d_dis = nullptr;
  float *d_t = nullptr;
  cudaMalloc(&d_ids, sizeof(int) * w * h);
  cudaMalloc(&d_t, sizeof(float) * w * h);
  cudaMalloc(&d_dis, sizeof(int));
  cudaMemset(d_dis, 0, sizeof(int));
  dim3 blk(32, 8), grd((w + 31) / 32, (h + 7) / 8);
  probe_kernel<<<grd, blk>>>(s->dev, w, h, (float)fr[0], (float)fr[1], (float)fr[2], (float)fr[3], (float)fr[4],
                             (float)fr[5], (float)fr[6], (float)fr[7], (float)fr[8], (float)fr[9], (float)fr[10],
                             (float)fr[11], d_ids, d_t, d_dis);
  cudaError_t e = cudaDeviceSynchronize();
  int dis = -1;
  if (e == cudaSuccess) {
    cudaMemcpy(ids_host, d_ids, sizeof(int) * w * h, cudaMemcpyDeviceToHost);
    cudaMemcpy(t_host, d_t, sizeof(float) * w * h, cudaMemcpyDeviceToHost);
    cudaMemcpy(&dis, d_dis, sizeof(int), cudaMemcpyDeviceToHost);
  }
  cudaFree(d_ids);
  cudaFree(d_t);
  cudaFree(d_dis);
  return e == cudaSuccess ? dis : -1000 - (int)e;
}

void refc_set_globals(float light, float background, float fuzz, float ior, int dof, float aperture, float focus) {
  setLightIntensity(light);
  setBackgroundIntensity(background);
  setMetalFuzziness(fuzz);
  setGlassRefractionIndex(ior);
  setDOFEnabled(dof != 0);
  setDOFAperture(aperture);
  setDOFFocusDistance(focus);
}

// As RendererCUDA::render (renderer_cuda_host.hpp:35-58): `chunks` accumulate
// calls of ~spp/chunks samples into a host float3 buffer. Returns seconds of
// wall time for the render loop (scene already resident), or < 0 on error.
double refc_render(void *sp, int w, int h, const double *fr, int spp, int chunks, int depth, float *accum) {
  auto *s = static_cast<RefGpuScene *>(sp);
  std::vector<float> buf((size_t)w * h * 3, 0.0f);
  void *d_rng = nullptr, *d_acc = nullptr;
  const int per = chunks > 0 ? (spp / chunks > 0 ? spp / chunks : 1) : spp;
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  int done = 0;
  while (done < spp) {
    const int add = per < spp - done ? per : spp - done;
    done += add;
    renderPixelsCUDAAccumulative(nullptr, buf.data(), s->dev, w, h, fr[0], fr[1], fr[2], fr[3], fr[4], fr[5], fr[6],
                                 fr[7], fr[8], fr[9], fr[10], fr[11], add, done, depth, &d_rng, &d_acc, fr[12],
                                 fr[13], fr[14], fr[15], fr[16], fr[17]);
  }
  cudaDeviceSynchronize();
  const auto t1 = std::chrono::steady_clock::now();
  if (accum) std::memcpy(accum, buf.data(), buf.size() * sizeof(float));
  if (d_rng) freeDeviceRandomStates(d_rng);
  if (d_acc) freeDeviceAccumBuffer(d_acc);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? std::chrono::duration<double>(t1 - t0).count() : -1.0;
}

// Device-resident variant (accum_buffer = nullptr, as the progressive
// renderer calls it, renderer_cuda_progressive_host.hpp:904): one call of spp
// samples timed with CUDA events; the sums stay on the device and are copied
// out afterwards (float4). Returns milliseconds.
float refc_render_device(void *sp, int w, int h, const double *fr, int spp, int depth, float *accum4) {
  auto *s = static_cast<RefGpuScene *>(sp);
  void *d_rng = nullptr, *d_acc = nullptr;
  // first call allocates and seeds; time a second one
  renderPixelsCUDAAccumulative(nullptr, nullptr, s->dev, w, h, fr[0], fr[1], fr[2], fr[3], fr[4], fr[5], fr[6],
                               fr[7], fr[8], fr[9], fr[10], fr[11], 1, 1, depth, &d_rng, &d_acc, fr[12], fr[13],
                               fr[14], fr[15], fr[16], fr[17]);
  resetDeviceAccumBuffer(d_acc, w * h);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a);
  renderPixelsCUDAAccumulative(nullptr, nullptr, s->dev, w, h, fr[0], fr[1], fr[2], fr[3], fr[4], fr[5], fr[6],
                               fr[7], fr[8], fr[9], fr[10], fr[11], spp, spp, depth, &d_rng, &d_acc, fr[12], fr[13],
                               fr[14], fr[15], fr[16], fr[17]);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  if (accum4) cudaMemcpy(accum4, d_acc, sizeof(float) * 4 * w * h, cudaMemcpyDeviceToHost);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  freeDeviceRandomStates(d_rng);
  freeDeviceAccumBuffer(d_acc);
  return cudaGetLastError() == cudaSuccess ? ms : -1.0f;
}

}  // extern "C"

// Scene construction (host) -------------------------------------------------
#include "rayon_b200_scene.h"
static Vec3 v3(const double *p) { return Vec3(p[0], p[1], p[2]); }

extern "C" void *refc_scene_create(const void *materials, int nmat, int mat_size, const uint8_t *kinds,
                                   const double *params, const int32_t *mats, int64_t n, int build_bvh) {
  if (mat_size != (int)sizeof(rb_material_desc)) return nullptr;
  auto *desc = new Scene::SceneDescription();
  const rb_material_desc *ms = static_cast<const rb_material_desc *>(materials);
  for (int i = 0; i < nmat; ++i) {
    const rb_material_desc *m = ms + i;
    Scene::MaterialDesc d;
    d.type = static_cast<Scene::MaterialType>(m->type);
    d.albedo = v3(m->albedo);
    d.emission = v3(m->emission);
    d.roughness = m->roughness;
    d.metallic = m->metallic;
    d.refractive_index = m->refractive_index;
    d.transmission = m->transmission;
    d.anisotropy = m->anisotropy;
    d.eta = v3(m->eta);
    d.k = v3(m->k);
    d.texture_id = m->texture_id;
    d.film_thickness = m->film_thickness;
    d.film_ior = m->film_ior;
    d.pattern = static_cast<Scene::ProceduralPattern>(m->pattern);
    d.pattern_color = v3(m->pattern_color);
    d.pattern_param1 = m->pattern_param1;
    d.pattern_param2 = m->pattern_param2;
    desc->addMaterial(d);
  }
  for (int64_t i = 0; i < n; ++i) {
    const double *p = params + 18 * i;
    switch (kinds[i]) {
      case 0: desc->addSphere(v3(p), p[3], mats[i]); break;
      case 1: desc->addRectangle(v3(p), v3(p + 3), v3(p + 6), mats[i]); break;
      case 2: desc->addTriangle(v3(p), v3(p + 3), v3(p + 6), mats[i]); break;
      default: break;
    }
  }
  if (build_bvh) desc->buildBVH();
  auto *s = new RefGpuScene{desc, Scene::CudaSceneBuilder::buildGPUScene(*desc)};
  return s;
}

// The reference's device scene pointer (CudaScene::Scene*), for calls into its
// own extern "C" renderer interface.
extern "C" void *refc_scene_device(void *sp) { return sp ? static_cast<RefGpuScene *>(sp)->dev : nullptr; }

extern "C" void refc_scene_destroy(void *sp) {
  auto *s = static_cast<RefGpuScene *>(sp);
  if (!s) return;
  Scene::CudaSceneBuilder::freeGPUScene(s->dev);
  delete s->desc;
  delete s;
}
