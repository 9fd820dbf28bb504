// Oracle infrastructure (test-only): RayON's own offline CUDA renderer,
// unmodified, running on librayon_b200.so.
//
// This translation unit includes the reference's RendererCUDA
// (src/rayon/gpu_renderers/renderer_cuda_host.hpp:23-74) and drives it the
// way RayON's main does, through RenderCoordinator::render
// (src/rayon/render/render_coordinator.cpp, compiled from its source) with a
// SceneDescription and a CameraBase. The library it is linked into
// (oracle/_ref/librayon_dropin.so, oracle/ref/Makefile) contains this file,
// render_coordinator.cpp and the adapter rayon_b200/adapter/rayon_b200_adapter.cpp,
// and no object of the reference's .cu sources: every CUDA entry point the
// renderer calls (renderPixelsCUDAAccumulative, freeDeviceRandomStates,
// freeDeviceAccumBuffer, setBackgroundIntensity, ...) and the scene upload
// resolve to librayon_b200.so. The link uses --no-undefined, so the build
// itself proves that every symbol resolves.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <vector>

#include "camera/camera_base.hpp"
#include "rayon_b200_scene.h"
#include "render/render_coordinator.hpp"
#include "renderer_cuda_host.hpp"
#include "scene_description.hpp"

namespace {
Vec3 v3(const double *p) { return Vec3(p[0], p[1], p[2]); }
}  // namespace

extern "C" {

// Builds the scene through SceneDescription (materials, then kinds 0 sphere,
// 1 rectangle, 2 triangle, 3 SDF primitive with 18 parameters each; buildBVH
// when build_bvh), sets the background intensity as a RayON caller does for a
// closed scene, and renders w x h at spp samples per pixel (depth 16, fixed by
// CameraBase) with RendererCUDA through RenderCoordinator::render at gamma
// 2.0. rgb receives the w*h*3 bytes the renderer writes into its target.
// Returns the ray count the renderer adds to the camera's counter.
long long dropin_render_offline(const rb_material_desc *mats, int nmat, const uint8_t *kinds, const double *params,
                                const int32_t *gmat, int64_t n, int build_bvh, const double *look_from,
                                const double *look_at, const double *vup, double vfov, int w, int h, int spp,
                                float background, unsigned char *rgb) {
  Scene::SceneDescription scene;
  for (int i = 0; i < nmat; ++i) {
    const rb_material_desc &m = mats[i];
    Scene::MaterialDesc d;
    d.type = static_cast<Scene::MaterialType>(m.type);
    d.albedo = v3(m.albedo);
    d.emission = v3(m.emission);
    d.roughness = m.roughness;
    d.metallic = m.metallic;
    d.refractive_index = m.refractive_index;
    d.transmission = m.transmission;
    d.anisotropy = m.anisotropy;
    d.eta = v3(m.eta);
    d.k = v3(m.k);
    d.texture_id = m.texture_id;
    d.film_thickness = m.film_thickness;
    d.film_ior = m.film_ior;
    d.pattern = static_cast<Scene::ProceduralPattern>(m.pattern);
    d.pattern_color = v3(m.pattern_color);
    d.pattern_param1 = m.pattern_param1;
    d.pattern_param2 = m.pattern_param2;
    scene.addMaterial(d);
  }
  for (int64_t i = 0; i < n; ++i) {
    const double *p = params + 18 * i;
    switch (kinds[i]) {
      case 0: scene.addSphere(v3(p), p[3], gmat[i]); break;
      case 1: scene.addRectangle(v3(p), v3(p + 3), v3(p + 6), gmat[i]); break;
      case 2: scene.addTriangle(v3(p), v3(p + 3), v3(p + 6), gmat[i]); break;
      case 3:
        scene.addSDFPrimitive(static_cast<Scene::SDFType>((int)p[0]), v3(p + 1), v3(p + 4), gmat[i], v3(p + 7));
        break;
      default: return -1;
    }
  }
  if (build_bvh) scene.buildBVH();
  CameraBase camera(Vec3(0, 0, 0), w, h, 3, spp, nullptr);
  camera.look_from = v3(look_from);
  camera.look_at = v3(look_at);
  camera.vup = v3(vup);
  camera.vfov = vfov;
  setBackgroundIntensity(background);
  RendererCUDA renderer;
  RenderCoordinator coordinator(camera, scene);
  std::vector<unsigned char> image;
  std::cout.setstate(std::ios::failbit);  // the renderer's progress bar
  coordinator.render(renderer, image, 2.0f);
  std::cout.clear();
  setBackgroundIntensity(1.0f);
  if (rgb) std::memcpy(rgb, image.data(), image.size());
  return camera.n_rays.load();
}

// The reference's host conversion of a float3 accumulation to bytes
// (render::convertAccumBufferToImage, render/render_utils.hpp:41-74), which
// RendererCUDA applies to its result.
void dropin_accum_to_image(const float *accum, int w, int h, int spp, float gamma, unsigned char *rgb) {
  std::vector<unsigned char> image((size_t)w * h * 3, 0);
  RenderTargetView target{&image, w, h, 3};
  std::vector<float> acc(accum, accum + (size_t)w * h * 3);
  render::convertAccumBufferToImage(target, acc, spp, gamma);
  std::memcpy(rgb, image.data(), image.size());
}

}  // extern "C"
