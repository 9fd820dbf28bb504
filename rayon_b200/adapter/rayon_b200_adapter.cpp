// rayon_b200_adapter.cpp -- the one translation unit a RayON maintainer adds to
// RayON's own tree so that its unmodified renderers run on this library.
//
// RayON's renderers (gpu_renderers/renderer_cuda_host.hpp:23-74,
// renderer_cuda_progressive_host.hpp) call two things: the extern "C"
// interface of gpu_renderers/renderer_cuda_device.cuh, which
// librayon_b200.so exports under the same names, and the C++ scene upload
// Scene::CudaSceneBuilder::{buildGPUScene, freeGPUScene}
// (scenes/scene_builder.hpp:234-239), which this file defines on top of the
// library's scene C-ABI. Compile it inside RayON against RayON's headers and
// link librayon_b200.so in place of the reference's .cu objects
// (renderer_cuda_device.cu, cuda_raytracer.cu, cuda_utils.cu,
// scene_builder_cuda.cu, shaders/*.cu).
//
// Scene conversion: every material and geometry of the SceneDescription goes
// through the library's builder calls, which keep the reference's bounds
// rules. When the description was built with a BVH (buildBVH, use_bvh true),
// the library builds its SAH BVH over the geometry in the description's
// (already leaf-ordered) sequence on all host cores. SDF primitives, which
// the reference's GPU path skips, are rendered.
#include <cstring>

#include "rayon_b200.h"
#include "scene_description.hpp"

namespace Scene {

// The class as scene_builder.hpp:234-239 declares it, declared here as the
// reference's own scene_builder_cuda.cu does: scene_builder.hpp pulls in the
// CPU shapes and data_structures/interval.hpp, whose static members are
// defined in the header and may be included by one translation unit only
// (RayON's main.cc).
class CudaSceneBuilder {
 public:
  static CudaScene::Scene *buildGPUScene(const SceneDescription &desc);
  static void freeGPUScene(CudaScene::Scene *scene);
};

namespace {
void put3(double *out, const Vec3 &v) {
  out[0] = v.x();
  out[1] = v.y();
  out[2] = v.z();
}
}  // namespace

CudaScene::Scene *CudaSceneBuilder::buildGPUScene(const SceneDescription &d) {
  rb_scene_desc *s = rb_scene_create();
  if (!s) return nullptr;
  for (const auto &m : d.materials) {
    rb_material_desc r;
    rb_material_default(&r);
    r.type = (int)m.type;
    put3(r.albedo, m.albedo);
    put3(r.emission, m.emission);
    r.roughness = m.roughness;
    r.metallic = m.metallic;
    r.refractive_index = m.refractive_index;
    r.transmission = m.transmission;
    r.anisotropy = m.anisotropy;
    put3(r.eta, m.eta);
    put3(r.k, m.k);
    r.texture_id = m.texture_id;
    r.film_thickness = m.film_thickness;
    r.film_ior = m.film_ior;
    r.pattern = (int)m.pattern;
    put3(r.pattern_color, m.pattern_color);
    r.pattern_param1 = m.pattern_param1;
    r.pattern_param2 = m.pattern_param2;
    rb_scene_add_material(s, &r);
  }
  bool has_sdf = false;
  for (const auto &g : d.geometries) {
    double a[3], b[3], c[3], n0[3], n1[3], n2[3];
    int idx = -1;
    switch (g.type) {
      case GeometryType::SPHERE:
        put3(a, g.data.sphere.center);
        idx = rb_scene_add_sphere(s, a, g.data.sphere.radius, g.material_id);
        break;
      case GeometryType::DISPLACED_SPHERE:
        put3(a, g.data.displaced_sphere.center);
        idx = rb_scene_add_displaced_sphere(s, a, g.data.displaced_sphere.radius, g.material_id,
                                            (float)g.data.displaced_sphere.displacement_scale,
                                            g.data.displaced_sphere.pattern_type);
        break;
      case GeometryType::RECTANGLE:
        put3(a, g.data.rectangle.corner);
        put3(b, g.data.rectangle.u);
        put3(c, g.data.rectangle.v);
        idx = rb_scene_add_rectangle(s, a, b, c, g.material_id);
        break;
      case GeometryType::TRIANGLE:
        put3(a, g.data.triangle.v0);
        put3(b, g.data.triangle.v1);
        put3(c, g.data.triangle.v2);
        if (g.data.triangle.has_normals) {
          put3(n0, g.data.triangle.n0);
          put3(n1, g.data.triangle.n1);
          put3(n2, g.data.triangle.n2);
          idx = rb_scene_add_triangle_with_normals(s, a, b, c, n0, n1, n2, g.material_id);
        } else {
          idx = rb_scene_add_triangle(s, a, b, c, g.material_id);
        }
        break;
      case GeometryType::SDF_PRIMITIVE:
        put3(a, g.data.sdf.position);
        put3(b, g.data.sdf.parameters);
        put3(c, g.data.sdf.rotation);
        idx = rb_scene_add_sdf(s, (int)g.data.sdf.sdf_type, a, b, c, g.material_id);
        has_sdf = true;
        break;
      default:  // cubes and mesh instances: the reference's GPU upload skips them too
        break;
    }
    if (idx >= 0 && !g.visible) rb_scene_set_visible(s, idx, 0);
  }
  // hard union, the reference CPU path's march settings (sdf.hpp:464-474)
  if (has_sdf) rb_scene_set_sdf_blend(s, 0.0f, 128, 1e-4f);
  if (d.use_bvh) rb_scene_build_bvh(s);
  rb_upload_opts o;
  std::memset(&o, 0, sizeof o);
  o.use_bvh = d.use_bvh ? 1 : 0;
  o.layout = RB_LAYOUT_AUTOTUNE;  // RB_LAYOUT_AS_BUILT keeps the built tree as is
  CudaScene::Scene *dev = rb_scene_upload(s, &o, nullptr);
  rb_scene_destroy(s);
  return dev;
}

void CudaSceneBuilder::freeGPUScene(CudaScene::Scene *scene) { rb_scene_free_device(scene); }

}  // namespace Scene
