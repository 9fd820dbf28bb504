// Host scene description (FP64) and SAH BVH builder of the B200 render path.
//
// Mirrors the builder interface and data semantics of Scene::SceneDescription
// (src/rayon/scenes/scene_description.hpp:445-925): the same bounds for every
// primitive kind, the same SAH BVH (node array, pre-order numbering, split
// choice, leaf-order geometry permutation). Storage is this project's own:
// one flat record per geometry and per-axis centroid keys for the sorts.
#pragma once

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/rayon_b200.h"

namespace rb {

struct V3 {
  double x = 0, y = 0, z = 0;
  V3() = default;
  V3(double a, double b, double c) : x(a), y(b), z(c) {}
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
// Vector algebra with the evaluation order of the reference's Vec3
// (data_structures/vec3.hpp:105-127): division is multiplication by 1/t.
inline V3 operator+(const V3 &a, const V3 &b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(const V3 &a, const V3 &b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(const V3 &a) { return V3(-a.x, -a.y, -a.z); }
inline V3 operator*(double t, const V3 &v) { return V3(t * v.x, t * v.y, t * v.z); }
inline V3 operator*(const V3 &v, double t) { return t * v; }
inline V3 operator/(const V3 &v, double t) { return (1 / t) * v; }
inline double dot(const V3 &a, const V3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(const V3 &u, const V3 &v) {
  return V3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
}
inline double length(const V3 &v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
inline V3 unit(const V3 &v) { return v / length(v); }

// One geometry. p[] holds the kind's parameters in FP64:
//   SPHERE / DISPLACED_SPHERE: p0-2 centre, p3 radius (p4 displacement, p5 pattern)
//   RECTANGLE: p0-2 corner, p3-5 u, p6-8 v
//   TRIANGLE:  p0-8 v0 v1 v2, p9-17 n0 n1 n2
//   SDF:       p0 sdf type, p1-3 position, p4-6 params, p7-9 rotation
struct Geom {
  uint8_t type = RB_GEOM_SPHERE;
  uint8_t visible = 1;
  uint8_t has_normals = 0;
  int32_t material_id = 0;
  double p[18] = {0};
  V3 bmin, bmax;
  int64_t orig = 0;  // insertion index
};

struct Node {
  double bmin[3], bmax[3];
  int32_t a = 0, b = 0;  // interior: left/right child; leaf: first geometry, count
  uint8_t is_leaf = 1, split_axis = 0;
};

struct SdfSettings {
  float blend_k = 0.0f;
  int max_steps = 256;
  float epsilon = 1e-4f;
};

class HostScene {
 public:
  std::vector<rb_material_desc> materials;
  std::vector<Geom> geoms;
  std::vector<Node> nodes;
  int root = -1;
  bool use_bvh = false;
  int max_leaf = 4;
  SdfSettings sdf;

  int add_material(const rb_material_desc &m);
  int64_t add_sphere(const V3 &c, double r, int mat);
  int64_t add_displaced_sphere(const V3 &c, double r, int mat, float disp, int pattern);
  int64_t add_rectangle(const V3 &corner, const V3 &u, const V3 &v, int mat);
  int64_t add_triangle(const V3 &v0, const V3 &v1, const V3 &v2, int mat);
  int64_t add_triangle_n(const V3 &v0, const V3 &v1, const V3 &v2, const V3 &n0, const V3 &n1,
                         const V3 &n2, int mat);
  int64_t add_sdf(int sdf_type, const V3 &pos, const V3 &params, const V3 &rot, int mat);

  // SAH build with the reference's split rule and ordering; returns false on
  // an empty scene (root = -1, as the reference).
  bool build_bvh(int max_leaf, int threads);
};

// Wavefront OBJ file into the scene with OBJLoader::loadOBJ's semantics
// (obj_ingest.cpp); returns the triangles added, or -1 with err set.
int64_t load_obj(HostScene &hs, const char *path, int mat, const V3 &pos, const V3 &scale, std::string &err);

// Radius of a sphere around an SDF primitive's position that contains it.
double sdf_bound_radius(const Geom &g);

// Camera frame (camera_base.hpp:76-99), FP64. out = 7 x 3 doubles.
void camera_frame(const V3 &look_from, const V3 &look_at, const V3 &vup, double vfov, int w, int h,
                  double out[21]);

void set_error(const std::string &msg);

}  // namespace rb
