// Oracle infrastructure (test-only): drives the reference's OWN host code,
// compiled from the unmodified sources under the reference tree (see
// oracle/ref/Makefile), for two purposes:
//   1. building a scene through Scene::SceneDescription's builder calls and
//      its buildBVH (src/rayon/scenes/scene_description.hpp:512-630, 717-925),
//      then exporting the node array and the leaf-order permutation, so the
//      project's BVH builder can be pinned against it bit for bit;
//   2. running the reference's multi-threaded CPU renderer RendererCPUParallel
//      (src/rayon/cpu_renderers/renderer_cpu_parallel.hpp:25-74) on the same
//      scene and camera as the timed CPU baseline;
//   3. the reference's camera frame (CameraBase::initialize / buildFrame,
//      src/rayon/camera/camera_base.hpp:47-99), so the project's camera frame
//      and the reference-arm renders use the reference's own numbers;
//   4. primary hits through the reference's CPU scene (CPUSceneBuilder,
//      src/rayon/scenes/scene_builder.hpp:46-80, and each shape's hit; SDF
//      primitives march in SDFShape::hit, cpu_shapes/sdf_shape.hpp:307-330,
//      with SDF::rayMarch, cpu_shapes/sdf.hpp:518-566), to pin the oracle's
//      SDF primitives.
// Nothing here is part of the product; only tests and bench.py's CPU-baseline
// leg load the resulting library.
#include <fcntl.h>
#include <unistd.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "rayon_b200_scene.h"
#include "camera/camera_base.hpp"
#include "render/renderer_interface.hpp"
#include "scene_builder.hpp"
#include "renderer_cpu_parallel.hpp"
#include "obj_loader.hpp"
#include "scene_description.hpp"

using Scene::SceneDescription;

namespace {
// Index of a geometry in insertion order, kept in a part of the geometry
// union that spheres, quads and normal-less triangles leave unused, so the
// leaf-order permutation can be read back after buildBVH.
void stash(Scene::GeometryDesc &g, int64_t i) { g.data.triangle.n2 = Vec3((double)i, 0.0, 0.0); }
int64_t unstash(const Scene::GeometryDesc &g) { return (int64_t)g.data.triangle.n2.x(); }
Vec3 v3(const double *p) { return Vec3(p[0], p[1], p[2]); }
}  // namespace

extern "C" {

void *refh_scene_create() { return new SceneDescription(); }
void refh_scene_destroy(void *s) { delete static_cast<SceneDescription *>(s); }

int refh_add_material(void *sp, const rb_material_desc *m) {
  auto *s = static_cast<SceneDescription *>(sp);
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
  return s->addMaterial(d);
}

// kinds: 0 sphere (c, r), 1 rectangle (corner, u, v), 2 triangle (v0, v1, v2),
// 3 SDF (type, position, params, rotation); params n x 18.
int refh_add_geoms(void *sp, const uint8_t *kinds, const double *params, const int32_t *mats, int64_t n) {
  auto *s = static_cast<SceneDescription *>(sp);
  for (int64_t i = 0; i < n; ++i) {
    const double *p = params + 18 * i;
    switch (kinds[i]) {
      case 0: s->addSphere(v3(p), p[3], mats[i]); break;
      case 1: s->addRectangle(v3(p), v3(p + 3), v3(p + 6), mats[i]); break;
      case 2: s->addTriangle(v3(p), v3(p + 3), v3(p + 6), mats[i]); break;
      case 3: s->addSDFPrimitive(static_cast<Scene::SDFType>((int)p[0]), v3(p + 1), v3(p + 4), mats[i], v3(p + 7)); break;
      default: return -1;
    }
    stash(s->geometries.back(), (int64_t)s->geometries.size() - 1);
  }
  return 0;
}

// The reference's OBJ loader (obj_loader.hpp:34-140) into the scene; returns its count or -1.
int refh_load_obj(void *sp, const char *path, int mat, const double *pos, const double *scale) {
  return Scene::OBJLoader::loadOBJ(path, *static_cast<SceneDescription *>(sp), mat, v3(pos), v3(scale));
}
int64_t refh_num_geoms(void *sp) { return (int64_t) static_cast<SceneDescription *>(sp)->geometries.size(); }
// Triangles in insertion order: v0 v1 v2 n0 n1 n2 (18 doubles), has_normals, material.
void refh_export_triangles(void *sp, double *out) {
  const auto &g = static_cast<SceneDescription *>(sp)->geometries;
  for (size_t i = 0; i < g.size(); ++i) {
    double *o = out + 20 * i;
    const auto &t = g[i].data.triangle;
    const Vec3 *v[6] = {&t.v0, &t.v1, &t.v2, &t.n0, &t.n1, &t.n2};
    for (int k = 0; k < 6; ++k)
      for (int c = 0; c < 3; ++c) o[3 * k + c] = (*v[k])[c];
    o[18] = t.has_normals ? 1.0 : 0.0;
    o[19] = (double)g[i].material_id;
  }
}

void refh_build_bvh(void *sp) { static_cast<SceneDescription *>(sp)->buildBVH(); }
int64_t refh_num_nodes(void *sp) { return (int64_t) static_cast<SceneDescription *>(sp)->top_level_bvh.nodes.size(); }
int refh_root(void *sp) { return static_cast<SceneDescription *>(sp)->top_level_bvh.root_index; }

void refh_export_bvh(void *sp, double *bounds, int32_t *a, int32_t *b, uint8_t *leaf, uint8_t *axis) {
  const auto &nodes = static_cast<SceneDescription *>(sp)->top_level_bvh.nodes;
  for (size_t i = 0; i < nodes.size(); ++i) {
    const auto &n = nodes[i];
    for (int k = 0; k < 3; ++k) {
      bounds[6 * i + k] = n.bounds_min[k];
      bounds[6 * i + 3 + k] = n.bounds_max[k];
    }
    a[i] = n.is_leaf ? n.data.leaf.first_geom_idx : n.data.interior.left_child;
    b[i] = n.is_leaf ? n.data.leaf.geom_count : n.data.interior.right_child;
    leaf[i] = n.is_leaf;
    axis[i] = n.split_axis;
  }
}

void refh_export_order(void *sp, int64_t *orig) {
  const auto &g = static_cast<SceneDescription *>(sp)->geometries;
  for (size_t i = 0; i < g.size(); ++i) orig[i] = unstash(g[i]);
}

// Renders with RendererCPUParallel (threads = hardware_concurrency, depth 16
// fixed by CameraBase::max_depth) and returns the wall time in seconds.
// Progress output is sent to /dev/null for the duration of the call.
double refh_render_cpu_parallel(void *sp, const double *look_from, const double *look_at, const double *vup,
                                double vfov, int w, int h, int spp, unsigned char *rgb_out, int *threads_used,
                                long long *rays_out) {
  auto *s = static_cast<SceneDescription *>(sp);
  CameraBase cam(Vec3(0, 0, 0), w, h, 3, spp, nullptr);
  cam.look_from = v3(look_from);
  cam.look_at = v3(look_at);
  cam.vup = v3(vup);
  cam.vfov = vfov;
  cam.updateFrame();
  std::vector<unsigned char> pixels((size_t)w * h * 3, 0);
  RenderTargetView target;
  target.pixels = &pixels;
  target.width = w;
  target.height = h;
  target.channels = 3;
  std::atomic<long long> counter{0};
  RenderContext ctx{counter, 2.0f};
  RenderRequest req{cam, *s, target};
  RendererCPUParallel r;
  fflush(stdout);
  const int saved = dup(1);
  const int devnull = open("/dev/null", O_WRONLY);
  dup2(devnull, 1);
  const auto t0 = std::chrono::steady_clock::now();
  r.render(req, ctx);
  const auto t1 = std::chrono::steady_clock::now();
  std::cout.flush();
  fflush(stdout);
  dup2(saved, 1);
  close(saved);
  close(devnull);
  if (rgb_out) std::memcpy(rgb_out, pixels.data(), pixels.size());
  if (threads_used) *threads_used = (int)std::max(1u, std::thread::hardware_concurrency());
  if (rays_out) *rays_out = counter.load();
  return std::chrono::duration<double>(t1 - t0).count();
}

// The reference's camera frame for (look_from, look_at, vup, vfov, w, h):
// out = camera_center, pixel00_loc, pixel_delta_u, pixel_delta_v, u, v, w
// (21 doubles), as CameraBase::buildFrame returns them after updateFrame.
void refh_camera_frame(const double *look_from, const double *look_at, const double *vup, double vfov, int w, int h,
                       double *out) {
  CameraBase cam(Vec3(0, 0, 0), w, h, 3, 1, nullptr);
  cam.look_from = v3(look_from);
  cam.look_at = v3(look_at);
  cam.vup = v3(vup);
  cam.vfov = vfov;
  cam.updateFrame();
  const CameraFrame f = cam.buildFrame();
  const Vec3 *v[7] = {&f.camera_center, &f.pixel00_loc, &f.pixel_delta_u, &f.pixel_delta_v, &f.u, &f.v, &f.w};
  for (int k = 0; k < 7; ++k)
    for (int c = 0; c < 3; ++c) out[3 * k + c] = (*v[k])[c];
}

// Pixel-centre primary rays (camera frame fr as above) through the
// reference's CPU scene: closest hit over its objects in order, exactly as
// Hittable_list::hit (data_structures/hittable_list.hpp:32-50) with
// Interval(0.001, +inf), recording which object was hit. The ray direction is
// normalised: SDF::rayMarch advances the ray parameter by the field value,
// which is a distance along the ray only for a unit direction. Outputs per
// pixel: object index or -1, t (a distance, since the direction is a unit
// vector), the recorded normal. Returns the number of objects in the scene.
int64_t refh_cpu_primary(void *sp, int w, int h, const double *fr, int32_t *ids, double *t_out, double *n_out) {
  auto *s = static_cast<SceneDescription *>(sp);
  const Hittable_list world = Scene::CPUSceneBuilder::buildCPUScene(*s);
  const Vec3 center(fr[0], fr[1], fr[2]), p00(fr[3], fr[4], fr[5]), du(fr[6], fr[7], fr[8]), dv(fr[9], fr[10], fr[11]);
  const int nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  auto work = [&](int tid) {
    for (int y = tid; y < h; y += nthreads)
      for (int x = 0; x < w; ++x) {
        const Vec3 pc = p00 + (double)x * du + (double)y * dv;
        const Ray r(center, unit_vector(pc - center));
        Hit_record tmp, rec;
        double closest = std::numeric_limits<double>::infinity();
        int hit = -1;
        for (size_t i = 0; i < world.objects.size(); ++i) {
          if (world.objects[i]->hit(r, Interval(0.001, closest), tmp)) {
            hit = (int)i;
            closest = tmp.t;
            rec = tmp;
          }
        }
        const size_t pix = (size_t)y * w + x;
        ids[pix] = hit;
        t_out[pix] = hit >= 0 ? rec.t : -1.0;
        for (int c = 0; c < 3; ++c) n_out[3 * pix + c] = hit >= 0 ? rec.normal[c] : 0.0;
      }
  };
  std::vector<std::thread> pool;
  for (int i = 0; i < nthreads; ++i) pool.emplace_back(work, i);
  for (auto &th : pool) th.join();
  return (int64_t)world.objects.size();
}

}  // extern "C"
