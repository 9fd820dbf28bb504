// Host scene description, SAH BVH builder and camera frame.
//
// The BVH follows SceneDescription::buildBVH / buildBVHRecursive
// (src/rayon/scenes/scene_description.hpp:717-778, 793-925):
//  - node bounds = union of the geometry boxes in the range (FP64);
//  - leaf when count <= max_leaf (the reference fixes 4, :817);
//  - for axis x, y, z in turn, std::sort the range by box centroid on that
//    axis, each sort starting from the previous order (:840-847), then an
//    O(n) prefix/suffix sweep evaluating cost = 1 + (A_L/A_P) i + (A_R/A_P)(n-i)
//    in FP32 with the areas rounded from FP64 (:849-899), first strict
//    minimum wins;
//  - a last std::sort on the winning axis (:902), node pushed in pre-order
//    before its children (:913-918);
//  - geometries permuted to leaf order (:736-777).
// Same sort algorithm (libstdc++ std::sort) and the same comparison outcomes
// give the same permutation, ties included. The sorts here run on packed
// (key, index) pairs for locality; std::sort's moves depend only on the
// comparison results, so the permutation is the one the reference's
// index sort produces. Subtrees are independent and are built on separate
// threads, then spliced in pre-order.
#include "host_scene.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <thread>

namespace rb {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }
const char *last_error_cstr() { return g_err.c_str(); }

int HostScene::add_material(const rb_material_desc &m) {
  materials.push_back(m);
  return (int)materials.size() - 1;
}

int64_t HostScene::add_sphere(const V3 &c, double r, int mat) {
  Geom g;
  g.type = RB_GEOM_SPHERE;
  g.material_id = mat;
  g.p[0] = c.x; g.p[1] = c.y; g.p[2] = c.z; g.p[3] = r;
  V3 rr(r, r, r);
  g.bmin = c - rr;
  g.bmax = c + rr;
  g.orig = (int64_t)geoms.size();
  geoms.push_back(g);
  return g.orig;
}

int64_t HostScene::add_displaced_sphere(const V3 &c, double r, int mat, float disp, int pattern) {
  Geom g;
  g.type = RB_GEOM_DISPLACED_SPHERE;
  g.material_id = mat;
  g.p[0] = c.x; g.p[1] = c.y; g.p[2] = c.z; g.p[3] = r;
  g.p[4] = disp; g.p[5] = pattern;
  V3 rr(r * 1.1, r * 1.1, r * 1.1);  // scene_description.hpp:538
  g.bmin = c - rr;
  g.bmax = c + rr;
  g.orig = (int64_t)geoms.size();
  geoms.push_back(g);
  return g.orig;
}

int64_t HostScene::add_rectangle(const V3 &corner, const V3 &u, const V3 &v, int mat) {
  Geom g;
  g.type = RB_GEOM_RECTANGLE;
  g.material_id = mat;
  const V3 vals[3] = {corner, u, v};
  for (int i = 0; i < 3; ++i) { g.p[3 * i] = vals[i].x; g.p[3 * i + 1] = vals[i].y; g.p[3 * i + 2] = vals[i].z; }
  // Box over the four corners (scene_description.hpp:553-573).
  const V3 cs[4] = {corner, corner + u, corner + v, corner + u + v};
  V3 lo = cs[0], hi = cs[0];
  for (int i = 1; i < 4; ++i) {
    lo = V3(std::min(lo.x, cs[i].x), std::min(lo.y, cs[i].y), std::min(lo.z, cs[i].z));
    hi = V3(std::max(hi.x, cs[i].x), std::max(hi.y, cs[i].y), std::max(hi.z, cs[i].z));
  }
  g.bmin = lo;
  g.bmax = hi;
  g.orig = (int64_t)geoms.size();
  geoms.push_back(g);
  return g.orig;
}

static void tri_box(Geom &g, const V3 &v0, const V3 &v1, const V3 &v2) {
  const double eps = 1e-4;  // zero-thickness padding (scene_description.hpp:588)
  g.bmin = V3(std::min(std::min(v0.x, v1.x), v2.x) - eps, std::min(std::min(v0.y, v1.y), v2.y) - eps,
              std::min(std::min(v0.z, v1.z), v2.z) - eps);
  g.bmax = V3(std::max(std::max(v0.x, v1.x), v2.x) + eps, std::max(std::max(v0.y, v1.y), v2.y) + eps,
              std::max(std::max(v0.z, v1.z), v2.z) + eps);
}

int64_t HostScene::add_triangle(const V3 &v0, const V3 &v1, const V3 &v2, int mat) {
  Geom g;
  g.type = RB_GEOM_TRIANGLE;
  g.material_id = mat;
  const V3 vs[3] = {v0, v1, v2};
  for (int i = 0; i < 3; ++i) { g.p[3 * i] = vs[i].x; g.p[3 * i + 1] = vs[i].y; g.p[3 * i + 2] = vs[i].z; }
  g.has_normals = 0;
  tri_box(g, v0, v1, v2);
  g.orig = (int64_t)geoms.size();
  geoms.push_back(g);
  return g.orig;
}

int64_t HostScene::add_triangle_n(const V3 &v0, const V3 &v1, const V3 &v2, const V3 &n0,
                                  const V3 &n1, const V3 &n2, int mat) {
  Geom g;
  g.type = RB_GEOM_TRIANGLE;
  g.material_id = mat;
  const V3 vs[6] = {v0, v1, v2, n0, n1, n2};
  for (int i = 0; i < 6; ++i) { g.p[3 * i] = vs[i].x; g.p[3 * i + 1] = vs[i].y; g.p[3 * i + 2] = vs[i].z; }
  g.has_normals = 1;
  tri_box(g, v0, v1, v2);
  g.orig = (int64_t)geoms.size();
  geoms.push_back(g);
  return g.orig;
}

int64_t HostScene::add_sdf(int sdf_type, const V3 &pos, const V3 &params, const V3 &rot, int mat) {
  Geom g;
  g.type = RB_GEOM_SDF_PRIMITIVE;
  g.material_id = mat;
  g.p[0] = sdf_type;
  g.p[1] = pos.x; g.p[2] = pos.y; g.p[3] = pos.z;
  g.p[4] = params.x; g.p[5] = params.y; g.p[6] = params.z;
  g.p[7] = rot.x; g.p[8] = rot.y; g.p[9] = rot.z;
  // The reference's placeholder box is pos -/+ params (scene_description.hpp:660-662);
  // that box does not contain a torus or capsule, so the device path bounds each
  // SDF primitive by its own conservative sphere at upload time instead.
  g.bmin = pos - params;
  g.bmax = pos + params;
  g.orig = (int64_t)geoms.size();
  geoms.push_back(g);
  return g.orig;
}

// ---------------------------------------------------------------------------
// SAH build
// ---------------------------------------------------------------------------
namespace {

struct Builder {
  const std::vector<Geom> &g;
  std::vector<int> idx;                  // geometry order, permuted in place
  std::vector<double> cent[3];           // centroid per axis, (bmin + bmax) * 0.5
  std::vector<double> box;               // 6 per geometry: bmin xyz, bmax xyz (compact copy)
  int max_leaf;

  explicit Builder(const std::vector<Geom> &geoms, int ml) : g(geoms), max_leaf(ml) {
    const size_t n = g.size();
    idx.resize(n);
    for (size_t i = 0; i < n; ++i) idx[i] = (int)i;
    for (int a = 0; a < 3; ++a) cent[a].resize(n);
    box.resize(6 * n);
    for (size_t i = 0; i < n; ++i) {
      const V3 c = (g[i].bmin + g[i].bmax) * 0.5;
      cent[0][i] = c.x; cent[1][i] = c.y; cent[2][i] = c.z;
      double *b = &box[6 * i];
      b[0] = g[i].bmin.x; b[1] = g[i].bmin.y; b[2] = g[i].bmin.z;
      b[3] = g[i].bmax.x; b[4] = g[i].bmax.y; b[5] = g[i].bmax.z;
    }
  }

  // Sorts idx[start, end) by centroid on `axis`; when sorted_boxes is given,
  // also writes the boxes of the range in the new order (6 doubles each), so
  // that the SAH sweeps read them sequentially.
  void sort_axis(int start, int end, int axis, std::vector<std::pair<double, int>> &buf,
                 std::vector<double> *sorted_boxes = nullptr) {
    const int n = end - start;
    buf.resize(n);
    const double *key = cent[axis].data();
    for (int i = 0; i < n; ++i) buf[i] = {key[idx[start + i]], idx[start + i]};
    std::sort(buf.begin(), buf.end(),
              [](const std::pair<double, int> &a, const std::pair<double, int> &b) {
                return a.first < b.first;
              });
    for (int i = 0; i < n; ++i) idx[start + i] = buf[i].second;
    if (sorted_boxes) {
      sorted_boxes->resize(6 * (size_t)n);
      double *o = sorted_boxes->data();
      for (int i = 0; i < n; ++i) std::memcpy(o + 6 * (size_t)i, &box[6 * (size_t)buf[i].second], 6 * sizeof(double));
    }
  }

  static float area_f(double ex, double ey, double ez) {
    // 2.0f * (FP64 expression), rounded to float on assignment (:833, :882-887).
    return (float)(2.0 * (ex * ey + ey * ez + ez * ex));
  }

  // Computes node bounds and, for an interior node, the split; leaves idx
  // sorted on the best axis. Returns the split index (or -1 for a leaf).
  int split(int start, int end, Node &node) {
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    for (int i = start; i < end; ++i) {
      const double *q = &box[6 * (size_t)idx[i]];
      lo[0] = std::min(lo[0], q[0]); lo[1] = std::min(lo[1], q[1]); lo[2] = std::min(lo[2], q[2]);
      hi[0] = std::max(hi[0], q[3]); hi[1] = std::max(hi[1], q[4]); hi[2] = std::max(hi[2], q[5]);
    }
    for (int a = 0; a < 3; ++a) { node.bmin[a] = lo[a]; node.bmax[a] = hi[a]; }
    const int count = end - start;
    if (count <= max_leaf) {
      node.is_leaf = 1;
      node.a = start;
      node.b = count;
      return -1;
    }
    float best_cost = 1e30f;
    int best_axis = 0;
    int best_split = start + count / 2;
    const float parent_area = area_f(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);

    thread_local std::vector<std::pair<double, int>> buf;
    thread_local std::vector<double> sb;  // the range's boxes in sorted order, 6 per entry
    thread_local std::vector<double> pmin, pmax, smin, smax;  // 3 per entry
    pmin.resize(3 * (size_t)count); pmax.resize(3 * (size_t)count);
    smin.resize(3 * (size_t)count); smax.resize(3 * (size_t)count);

    for (int axis = 0; axis < 3; ++axis) {
      sort_axis(start, end, axis, buf, &sb);
      double rl[3] = {1e30, 1e30, 1e30}, rh[3] = {-1e30, -1e30, -1e30};
      for (int i = 0; i < count; ++i) {
        const double *q = &sb[6 * (size_t)i];
        rl[0] = std::min(rl[0], q[0]); rl[1] = std::min(rl[1], q[1]); rl[2] = std::min(rl[2], q[2]);
        rh[0] = std::max(rh[0], q[3]); rh[1] = std::max(rh[1], q[4]); rh[2] = std::max(rh[2], q[5]);
        std::memcpy(&pmin[3 * i], rl, sizeof rl);
        std::memcpy(&pmax[3 * i], rh, sizeof rh);
      }
      rl[0] = rl[1] = rl[2] = 1e30;
      rh[0] = rh[1] = rh[2] = -1e30;
      for (int i = count - 1; i >= 0; --i) {
        const double *q = &sb[6 * (size_t)i];
        rl[0] = std::min(rl[0], q[0]); rl[1] = std::min(rl[1], q[1]); rl[2] = std::min(rl[2], q[2]);
        rh[0] = std::max(rh[0], q[3]); rh[1] = std::max(rh[1], q[4]); rh[2] = std::max(rh[2], q[5]);
        std::memcpy(&smin[3 * i], rl, sizeof rl);
        std::memcpy(&smax[3 * i], rh, sizeof rh);
      }
      for (int i = 1; i < count; ++i) {
        const double *a0 = &pmin[3 * (i - 1)], *a1 = &pmax[3 * (i - 1)];
        const double *b0 = &smin[3 * i], *b1 = &smax[3 * i];
        const float la = area_f(a1[0] - a0[0], a1[1] - a0[1], a1[2] - a0[2]);
        const float ra = area_f(b1[0] - b0[0], b1[1] - b0[1], b1[2] - b0[2]);
        const float cost = 1.0f + (la / parent_area) * (float)i + (ra / parent_area) * (float)(count - i);
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = axis;
          best_split = start + i;
        }
      }
    }
    sort_axis(start, end, best_axis, buf);
    node.is_leaf = 0;
    node.split_axis = (uint8_t)best_axis;
    return best_split;
  }

  // Serial pre-order build appending to out.
  int build_serial(int start, int end, std::vector<Node> &out) {
    Node node;
    const int s = split(start, end, node);
    const int me = (int)out.size();
    out.push_back(node);
    if (s < 0) return me;
    const int l = build_serial(start, s, out);
    const int r = build_serial(s, end, out);
    out[me].a = l;
    out[me].b = r;
    return me;
  }

  static void shift(std::vector<Node> &v, int off) {
    for (auto &n : v)
      if (!n.is_leaf) { n.a += off; n.b += off; }
  }

  // Parallel build of [start, end) into a pre-order vector rooted at index 0.
  std::vector<Node> build_par(int start, int end, int depth, int par_depth) {
    std::vector<Node> out;
    if (depth >= par_depth || end - start < 4096) {
      build_serial(start, end, out);
      return out;
    }
    Node node;
    const int s = split(start, end, node);
    if (s < 0) {
      out.push_back(node);
      return out;
    }
    auto fl = std::async(std::launch::async, [&]() { return build_par(start, s, depth + 1, par_depth); });
    std::vector<Node> R = build_par(s, end, depth + 1, par_depth);
    std::vector<Node> L = fl.get();
    out.reserve(1 + L.size() + R.size());
    node.a = 1;
    node.b = 1 + (int)L.size();
    out.push_back(node);
    shift(L, 1);
    shift(R, 1 + (int)L.size());
    out.insert(out.end(), L.begin(), L.end());
    out.insert(out.end(), R.begin(), R.end());
    return out;
  }
};

}  // namespace

double sdf_bound_radius(const Geom &g) {
  const double a = std::fabs(g.p[4]), b = std::fabs(g.p[5]), c = std::fabs(g.p[6]);
  switch ((int)g.p[0]) {
    case RB_SDF_SPHERE: return a;
    case RB_SDF_BOX:
    case RB_SDF_ROUND_BOX: return std::sqrt(a * a + b * b + c * c);
    case RB_SDF_TORUS: return a + b;
    case RB_SDF_CAPSULE: return a + 0.5 * b;
    default: return std::max(a, std::max(b, c));
  }
}

bool HostScene::build_bvh(int leaf, int threads) {
  nodes.clear();
  // SDF primitives are bounded by their own sphere grown by the smooth-union
  // radius (the reference's pos -/+ params box does not contain tori or
  // capsules, and blended surfaces reach up to k further)
  for (Geom &g : geoms)
    if (g.type == RB_GEOM_SDF_PRIMITIVE) {
      const double r = sdf_bound_radius(g) * 1.0001 + sdf.blend_k + 1e-3;
      const V3 c(g.p[1], g.p[2], g.p[3]);
      g.bmin = c - V3(r, r, r);
      g.bmax = c + V3(r, r, r);
    }
  if (geoms.empty()) {
    root = -1;
    return false;
  }
  use_bvh = true;
  max_leaf = leaf;
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  int par_depth = 0;
  while ((1 << par_depth) < 2 * threads && par_depth < 12) ++par_depth;
  if (threads == 1) par_depth = 0;
  Builder b(geoms, leaf);
  nodes = b.build_par(0, (int)geoms.size(), 0, par_depth);
  root = 0;
  // Leaf order: the DFS left-then-right order of leaves is the order of their
  // ranges, so the permuted array is geoms[idx[i]] and every leaf keeps its
  // first index (scene_description.hpp:736-777).
  std::vector<Geom> re(geoms.size());
  for (size_t i = 0; i < geoms.size(); ++i) re[i] = geoms[b.idx[i]];
  geoms.swap(re);
  return true;
}

void camera_frame(const V3 &from, const V3 &at, const V3 &vup, double vfov, int width, int height,
                  double out[21]) {
  const V3 center = from;
  const double focal = length(from - at);
  const double theta = vfov * M_PI / 180.0;
  const double h = std::tan(theta / 2);
  const double vh = 2 * h * focal;
  const double vw = vh * (double(width) / height);
  const V3 w = unit(from - at);
  const V3 u = unit(cross(vup, w));
  const V3 v = cross(w, u);
  const V3 vu = vw * u;
  const V3 vv = vh * -v;
  const V3 du = vu / width;
  const V3 dv = vv / height;
  const V3 upper_left = center - (focal * w) - vu / 2 - vv / 2;
  const V3 p00 = upper_left + 0.5 * (du + dv);
  const V3 vals[7] = {center, p00, du, dv, u, v, w};
  for (int i = 0; i < 7; ++i) { out[3 * i] = vals[i].x; out[3 * i + 1] = vals[i].y; out[3 * i + 2] = vals[i].z; }
}

}  // namespace rb
