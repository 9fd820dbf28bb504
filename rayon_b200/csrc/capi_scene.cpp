// C-ABI over the host scene description (section 2 of rayon_b200.h).
#include <cstring>
#include <exception>

#include "host_scene.hpp"

namespace rb {
const char *last_error_cstr();
}

struct rb_scene_desc {
  rb::HostScene s;
};

using rb::V3;

static V3 v3(const double *p) { return V3(p[0], p[1], p[2]); }

extern "C" {

const char *rb_last_error(void) { return rb::last_error_cstr(); }
const char *rb_version(void) { return "rayon_b200 0.1.0 (sm_100a)"; }

void rb_material_default(rb_material_desc *m) {
  // MaterialDesc() defaults (scene_description.hpp:83-101).
  std::memset(m, 0, sizeof *m);
  m->type = RB_MAT_LAMBERTIAN;
  m->albedo[0] = m->albedo[1] = m->albedo[2] = 0.7;
  m->roughness = 0.0f;
  m->metallic = 0.0f;
  m->refractive_index = 1.0f;
  m->transmission = 0.0f;
  m->anisotropy = 0.0f;
  m->texture_id = -1;
  m->film_thickness = 400.0f;
  m->film_ior = 1.33f;
  m->pattern = 0;
}

rb_scene_desc *rb_scene_create(void) {
  try {
    return new rb_scene_desc();
  } catch (const std::exception &e) {
    rb::set_error(e.what());
    return nullptr;
  }
}
void rb_scene_destroy(rb_scene_desc *s) { delete s; }

int rb_scene_add_material(rb_scene_desc *s, const rb_material_desc *m) {
  if (!s || !m) { rb::set_error("rb_scene_add_material: null argument"); return RB_ERR_INVALID_ARG; }
  return s->s.add_material(*m);
}

int rb_scene_add_sphere(rb_scene_desc *s, const double c[3], double r, int mat) {
  if (!s || !c) return RB_ERR_INVALID_ARG;
  return (int)s->s.add_sphere(v3(c), r, mat);
}

int rb_scene_add_displaced_sphere(rb_scene_desc *s, const double c[3], double r, int mat, float disp,
                                  int pattern) {
  if (!s || !c) return RB_ERR_INVALID_ARG;
  return (int)s->s.add_displaced_sphere(v3(c), r, mat, disp, pattern);
}

int rb_scene_add_rectangle(rb_scene_desc *s, const double corner[3], const double u[3],
                           const double v[3], int mat) {
  if (!s || !corner || !u || !v) return RB_ERR_INVALID_ARG;
  return (int)s->s.add_rectangle(v3(corner), v3(u), v3(v), mat);
}

int rb_scene_add_triangle(rb_scene_desc *s, const double v0[3], const double v1[3],
                          const double v2[3], int mat) {
  if (!s || !v0 || !v1 || !v2) return RB_ERR_INVALID_ARG;
  return (int)s->s.add_triangle(v3(v0), v3(v1), v3(v2), mat);
}

int rb_scene_add_triangle_with_normals(rb_scene_desc *s, const double v0[3], const double v1[3],
                                       const double v2[3], const double n0[3], const double n1[3],
                                       const double n2[3], int mat) {
  if (!s || !v0 || !v1 || !v2 || !n0 || !n1 || !n2) return RB_ERR_INVALID_ARG;
  return (int)s->s.add_triangle_n(v3(v0), v3(v1), v3(v2), v3(n0), v3(n1), v3(n2), mat);
}

int rb_scene_add_sdf(rb_scene_desc *s, int sdf_type, const double pos[3], const double params[3],
                     const double rot[3], int mat) {
  if (!s || !pos || !params) return RB_ERR_INVALID_ARG;
  const double zero[3] = {0, 0, 0};
  return (int)s->s.add_sdf(sdf_type, v3(pos), v3(params), v3(rot ? rot : zero), mat);
}

int64_t rb_scene_add_spheres(rb_scene_desc *s, const double *cr, const int32_t *mats, int mat,
                             int64_t n) {
  if (!s || (!cr && n > 0) || n < 0) return RB_ERR_INVALID_ARG;
  const int64_t first = (int64_t)s->s.geoms.size();
  s->s.geoms.reserve(first + n);
  for (int64_t i = 0; i < n; ++i)
    s->s.add_sphere(v3(cr + 4 * i), cr[4 * i + 3], mats ? mats[i] : mat);
  return first;
}

int64_t rb_scene_add_triangles(rb_scene_desc *s, const double *v, const double *nrm,
                               const int32_t *mats, int mat, int64_t n) {
  if (!s || (!v && n > 0) || n < 0) return RB_ERR_INVALID_ARG;
  const int64_t first = (int64_t)s->s.geoms.size();
  s->s.geoms.reserve(first + n);
  for (int64_t i = 0; i < n; ++i) {
    const double *p = v + 9 * i;
    const int m = mats ? mats[i] : mat;
    if (nrm) {
      const double *q = nrm + 9 * i;
      s->s.add_triangle_n(v3(p), v3(p + 3), v3(p + 6), v3(q), v3(q + 3), v3(q + 6), m);
    } else {
      s->s.add_triangle(v3(p), v3(p + 3), v3(p + 6), m);
    }
  }
  return first;
}

int64_t rb_scene_load_obj(rb_scene_desc *s, const char *path, int mat_id, const double position[3],
                          const double scale[3]) {
  if (!s || !path) return RB_ERR_INVALID_ARG;
  const V3 pos = position ? v3(position) : V3(0, 0, 0);
  const V3 sc = scale ? v3(scale) : V3(1, 1, 1);
  std::string err;
  const int64_t n = rb::load_obj(s->s, path, mat_id, pos, sc, err);
  if (n < 0) {
    rb::set_error("rb_scene_load_obj: " + err);
    return err.rfind("cannot open", 0) == 0 ? RB_ERR_NOT_FOUND : RB_ERR_INVALID_ARG;
  }
  return n;
}

int rb_scene_set_visible(rb_scene_desc *s, int64_t i, int visible) {
  // i is the insertion index (the index an add call returned), also after a
  // BVH build has permuted the geometries to leaf order.
  if (!s || i < 0 || i >= (int64_t)s->s.geoms.size()) {
    rb::set_error("rb_scene_set_visible: geometry index out of range");
    return RB_ERR_INVALID_ARG;
  }
  auto &g = s->s.geoms;
  if (g[i].orig != i) {
    for (auto &q : g)
      if (q.orig == i) {
        q.visible = visible ? 1 : 0;
        return RB_OK;
      }
  }
  g[i].visible = visible ? 1 : 0;
  return RB_OK;
}

int64_t rb_scene_num_geometries(const rb_scene_desc *s) { return s ? (int64_t)s->s.geoms.size() : 0; }
int rb_scene_num_materials(const rb_scene_desc *s) { return s ? (int)s->s.materials.size() : 0; }

int rb_scene_set_sdf_blend(rb_scene_desc *s, float k, int max_steps, float eps) {
  if (!s || k < 0 || max_steps <= 0 || eps <= 0) return RB_ERR_INVALID_ARG;
  s->s.sdf.blend_k = k;
  s->s.sdf.max_steps = max_steps;
  s->s.sdf.epsilon = eps;
  return RB_OK;
}

int rb_scene_build_bvh(rb_scene_desc *s) { return rb_scene_build_bvh_ex(s, 4, 0); }

int rb_scene_build_bvh_ex(rb_scene_desc *s, int max_leaf, int threads) {
  if (!s || max_leaf < 1 || max_leaf > 32) {
    rb::set_error("rb_scene_build_bvh_ex: max_leaf must be in [1, 32]");
    return RB_ERR_INVALID_ARG;
  }
  if (s->s.geoms.size() >= (size_t)(1u << 27)) {
    rb::set_error("rb_scene_build_bvh_ex: more than 2^27 geometries");
    return RB_ERR_CAPACITY;
  }
  try {
    s->s.build_bvh(max_leaf, threads);
  } catch (const std::exception &e) {
    rb::set_error(std::string("rb_scene_build_bvh_ex: ") + e.what());
    return RB_ERR_OUT_OF_MEMORY;
  }
  return RB_OK;
}

int64_t rb_scene_num_bvh_nodes(const rb_scene_desc *s) { return s ? (int64_t)s->s.nodes.size() : 0; }
int rb_scene_bvh_root(const rb_scene_desc *s) { return s ? s->s.root : -1; }

int rb_scene_export_bvh(const rb_scene_desc *s, double *bounds, int32_t *a, int32_t *b,
                        uint8_t *is_leaf, uint8_t *axis) {
  if (!s) return RB_ERR_INVALID_ARG;
  const auto &nodes = s->s.nodes;
  for (size_t i = 0; i < nodes.size(); ++i) {
    const rb::Node &n = nodes[i];
    if (bounds) {
      for (int k = 0; k < 3; ++k) { bounds[6 * i + k] = n.bmin[k]; bounds[6 * i + 3 + k] = n.bmax[k]; }
    }
    if (a) a[i] = n.a;
    if (b) b[i] = n.b;
    if (is_leaf) is_leaf[i] = n.is_leaf;
    if (axis) axis[i] = n.split_axis;
  }
  return RB_OK;
}

int rb_scene_export_order(const rb_scene_desc *s, int64_t *orig) {
  if (!s || !orig) return RB_ERR_INVALID_ARG;
  for (size_t i = 0; i < s->s.geoms.size(); ++i) orig[i] = s->s.geoms[i].orig;
  return RB_OK;
}

int rb_scene_export_geometry_full(const rb_scene_desc *s, double *out) {
  if (!s || !out) return RB_ERR_INVALID_ARG;
  for (size_t i = 0; i < s->s.geoms.size(); ++i) {
    const rb::Geom &g = s->s.geoms[i];
    double *o = out + 32 * i;
    o[0] = g.type; o[1] = g.material_id; o[2] = g.visible; o[3] = g.has_normals;
    for (int k = 0; k < 18; ++k) o[4 + k] = g.p[k];
    o[22] = g.bmin.x; o[23] = g.bmin.y; o[24] = g.bmin.z;
    o[25] = g.bmax.x; o[26] = g.bmax.y; o[27] = g.bmax.z;
    o[28] = (double)g.orig; o[29] = o[30] = o[31] = 0;
  }
  return RB_OK;
}

int rb_scene_export_materials(const rb_scene_desc *s, rb_material_desc *out) {
  if (!s || !out) return RB_ERR_INVALID_ARG;
  for (size_t i = 0; i < s->s.materials.size(); ++i) out[i] = s->s.materials[i];
  return RB_OK;
}

void rb_camera_frame(const double from[3], const double at[3], const double vup[3], double vfov,
                     int w, int h, double out[21]) {
  rb::camera_frame(v3(from), v3(at), v3(vup), vfov, w, h, out);
}

}  // extern "C"

// Host-side access for the device translation units.
namespace rb {
const HostScene &host_scene_of(const rb_scene_desc *s) { return s->s; }
}
