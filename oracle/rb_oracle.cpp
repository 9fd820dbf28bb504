// FP64 CPU oracle of the RayON GPU render path -- TEST INFRASTRUCTURE ONLY.
//
// A double-precision restatement of the reference's CUDA path tracer,
// following src/rayon/gpu_renderers/cuda_raytracer.cuh:
//   hit_aabb :154-197, hit_sphere :203-233, hit_rectangle :235-271,
//   hit_triangle :277-347, hit_scene (closest hit, DFS near-first by split
//   axis sign, equal-t later-wins rule) :487-602, apply_material :418-485,
//   scatter_material :613-850, ray_color (bounce loop, invisible-at-bounce-0,
//   Russian roulette from bounce 1, sky) :858-933;
// microfacet_ggx.cuh:21-111; render_acc_kernel.cu:198-238 (camera ray, DOF);
// camera_base.hpp:76-99 (frame, supplied by the caller).
// Random numbers come from rb_rng.h, the same counter-based streams the CUDA
// kernels use, so each path is paired with the GPU's and the comparison is
// per path, not only statistical. Next-event estimation (not in the
// reference) is restated from the CUDA path with the same MIS weights.
//
// The product path never links or calls this file; only tests/, the smoke
// check and bench.py's CPU-baseline leg do.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/rayon_b200_scene.h"
#include "../rayon_b200/csrc/rb_rng.h"

namespace {

struct D3 {
  double x = 0, y = 0, z = 0;
  D3() = default;
  D3(double a, double b, double c) : x(a), y(b), z(c) {}
  D3 operator+(const D3 &o) const { return D3(x + o.x, y + o.y, z + o.z); }
  D3 operator-(const D3 &o) const { return D3(x - o.x, y - o.y, z - o.z); }
  D3 operator*(double t) const { return D3(x * t, y * t, z * t); }
  D3 operator*(const D3 &o) const { return D3(x * o.x, y * o.y, z * o.z); }
  D3 operator/(double t) const { return D3(x / t, y / t, z / t); }
  D3 operator-() const { return D3(-x, -y, -z); }
  double len2() const { return x * x + y * y + z * z; }
  double len() const { return std::sqrt(len2()); }
};
D3 operator*(double t, const D3 &v) { return v * t; }
double dot(const D3 &a, const D3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
D3 cross(const D3 &a, const D3 &b) { return D3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
D3 norm(const D3 &v) { return v / v.len(); }

const double PI = 3.14159265358979323846;

struct Ray {
  D3 o, d;
  D3 at(double t) const { return o + t * d; }
};

enum { L_LAMB = 0, L_MIRROR = 1, L_GLASS = 2, L_LIGHT = 3, L_ROUGH = 4, L_CONST = 5, L_NORMALS = 6, L_ANISO = 7,
       L_FILM = 8, L_COAT = 9, L_ABSORB = 15 };

struct Mat {
  int kind, pattern;
  D3 color, emission, eta, k, pattern_color;
  double roughness, ior, anisotropy, film_thickness, film_ior, p1, p2;
};

struct Geom {
  int type, mat, visible, has_normals;
  double p[18];
};

struct Node {
  double lo[3], hi[3];
  int a, b, leaf, axis;
};

struct Globals {
  double light, background, fuzz, glass_ior;
  int dof;
  double aperture, focus;
  int nee;
};

struct Light {
  int prim;
  double area, cdf;
};

struct SdfP {
  int type, mat;
  D3 pos;
  double a, b, c, round, bound;
  double R[9];  // world -> local
};

struct Scene {
  std::vector<Geom> g;
  std::vector<Mat> m;
  std::vector<Node> n;
  std::vector<Light> lights;
  double light_area = 0;
  int root = -1;
  std::vector<SdfP> sdf;        // SDF primitives in geometry (leaf) order
  std::vector<int> sdf_of_geom; // geometry index -> sdf index or -1
  double sdf_k = 0;
  int sdf_steps = 256;
  double sdf_eps = 1e-4;
};

// Work counters. kind[] counts primitive tests by geometry kind (sphere and
// displaced sphere, rectangle, triangle, SDF primitive); shade[] counts
// shading events by resolved material class (Lambert, mirror and rough
// mirror, glass, light and constant and normals, GGX conductor / thin film /
// clear coat).
struct Counters {
  int64_t nodes = 0, prims = 0, segments = 0, paths = 0, shadow = 0;
  int64_t kind[4] = {0, 0, 0, 0};
  int64_t shade[5] = {0, 0, 0, 0, 0};
};
enum { ORC_NCOUNTERS = 14 };

Mat resolve(const rb_material_desc &d) {
  Mat m;
  std::memset(&m, 0, sizeof m);
  auto v = [](const double *p) { return D3(p[0], p[1], p[2]); };
  m.color = v(d.albedo);
  m.emission = v(d.emission);
  m.eta = v(d.eta);
  m.k = v(d.k);
  m.pattern_color = v(d.pattern_color);
  m.roughness = d.roughness;
  m.ior = d.refractive_index;
  m.anisotropy = d.anisotropy;
  m.film_thickness = d.film_thickness;
  m.film_ior = d.film_ior;
  m.pattern = d.pattern == 1;
  m.p1 = d.pattern_param1;
  m.p2 = d.pattern_param2;
  switch (d.type) {
    case RB_MAT_LAMBERTIAN: case RB_MAT_SDF_MATERIAL: m.kind = L_LAMB; break;
    case RB_MAT_MIRROR: m.kind = L_MIRROR; break;
    case RB_MAT_METAL: case RB_MAT_ROUGH_MIRROR:
      m.kind = L_ROUGH;
      m.roughness = d.roughness > 0.0f ? d.roughness : 0.3f;
      break;
    case RB_MAT_GLASS: case RB_MAT_DIELECTRIC: m.kind = L_GLASS; break;
    case RB_MAT_LIGHT: m.kind = L_LIGHT; break;
    case RB_MAT_CONSTANT: m.kind = L_CONST; break;
    case RB_MAT_SHOW_NORMALS: m.kind = L_NORMALS; break;
    case RB_MAT_ANISOTROPIC_METAL: m.kind = L_ANISO; break;
    case RB_MAT_THIN_FILM: m.kind = L_FILM; break;
    case RB_MAT_CLEAR_COAT:
      m.kind = L_COAT;
      m.ior = d.refractive_index > 1.0f ? d.refractive_index : 1.5f;
      break;
    default: m.kind = L_ABSORB;
  }
  return m;
}

// --- primitives (FP64) --------------------------------------------------------
bool box_hit(const Ray &r, const double *lo, const double *hi, double tmin, double tmax) {
  double te = -INFINITY, tx = INFINITY;
  double t0[3], t1[3];
  const double o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
  for (int k = 0; k < 3; ++k) {
    const double inv = 1.0 / d[k];
    double a = (lo[k] - o[k]) * inv, b = (hi[k] - o[k]) * inv;
    if (inv < 0.0) std::swap(a, b);
    t0[k] = a;
    t1[k] = b;
  }
  te = std::fmax(std::fmax(t0[0], t0[1]), t0[2]);
  tx = std::fmin(std::fmin(t1[0], t1[1]), t1[2]);
  return te <= tx && tx >= tmin && te <= tmax;
}

bool t_sphere(const D3 &c, double rad, const Ray &r, double tmin, double tmax, double &t) {
  const D3 oc = r.o - c;
  const double a = dot(r.d, r.d), hb = dot(oc, r.d), cc = dot(oc, oc) - rad * rad;
  const double disc = hb * hb - a * cc;
  if (disc < 0) return false;
  const double sq = std::sqrt(disc);
  double root = (-hb - sq) / a;
  if (root < tmin || tmax < root) {
    root = (-hb + sq) / a;
    if (root < tmin || tmax < root) return false;
  }
  t = root;
  return true;
}

bool t_rect(const D3 &corner, const D3 &u, const D3 &v, const Ray &r, double tmin, double tmax, double &tt) {
  const D3 n = norm(cross(u, v));
  const double den = dot(n, r.d);
  if (std::fabs(den) < 1e-8) return false;
  const double t = dot(n, corner - r.o) / den;
  if (t < tmin || t > tmax) return false;
  const D3 p = r.at(t) - corner;
  const double al = dot(p, u) / dot(u, u), be = dot(p, v) / dot(v, v);
  if (al < 0 || al > 1 || be < 0 || be > 1) return false;
  tt = t;
  return true;
}

bool t_tri(const D3 &v0, const D3 &v1, const D3 &v2, const Ray &r, double tmin, double tmax, double &tt) {
  const D3 e1 = v1 - v0, e2 = v2 - v0;
  const D3 h = cross(r.d, e2);
  const double a = dot(e1, h);
  if (std::fabs(a) < 1e-8) return false;
  const double f = 1.0 / a;
  const D3 s = r.o - v0;
  const double u = f * dot(s, h);
  if (u < 0 || u > 1) return false;
  const D3 q = cross(s, e1);
  const double v = f * dot(r.d, q);
  if (v < 0 || u + v > 1) return false;
  const double t = f * dot(e2, q);
  if (t < tmin || t > tmax) return false;
  tt = t;
  return true;
}

D3 gv(const Geom &g, int i) { return D3(g.p[i], g.p[i + 1], g.p[i + 2]); }

// SDF distance functions (cpu_shapes/sdf.hpp:105-160; rounded box = box of
// half extents minus the rounding radius, grown by it), evaluated in the
// primitive's local frame.
double sdf_eval1(const SdfP &q, const D3 &pw) {
  const D3 d0 = pw - q.pos;
  const D3 p(q.R[0] * d0.x + q.R[1] * d0.y + q.R[2] * d0.z, q.R[3] * d0.x + q.R[4] * d0.y + q.R[5] * d0.z,
             q.R[6] * d0.x + q.R[7] * d0.y + q.R[8] * d0.z);
  switch (q.type) {
    case RB_SDF_SPHERE: return p.len() - q.a;
    case RB_SDF_BOX:
    case RB_SDF_ROUND_BOX: {
      const D3 qq(std::fabs(p.x) - (q.a - q.round), std::fabs(p.y) - (q.b - q.round), std::fabs(p.z) - (q.c - q.round));
      const double out = D3(std::fmax(qq.x, 0.0), std::fmax(qq.y, 0.0), std::fmax(qq.z, 0.0)).len();
      const double in = std::fmin(std::fmax(qq.x, std::fmax(qq.y, qq.z)), 0.0);
      return out + in - q.round;
    }
    case RB_SDF_TORUS: {
      const double qx = std::sqrt(p.x * p.x + p.z * p.z) - q.a;
      return std::sqrt(qx * qx + p.y * p.y) - q.b;
    }
    case RB_SDF_CAPSULE: {
      const double hh = q.b * 0.5, y = std::fmin(std::fmax(p.y, -hh), hh);
      return D3(p.x, p.y - y, p.z).len() - q.a;
    }
    default: return 1e30;
  }
}

// polynomial smooth minimum (sdf.hpp:410-416)
double smin_poly(double d1, double d2, double k) {
  const double h = std::fmin(std::fmax(0.5 + 0.5 * (d2 - d1) / k, 0.0), 1.0);
  return d2 * (1.0 - h) + d1 * h - k * h * (1.0 - h);
}

double inflated_radius(const Scene &S, const SdfP &q) { return q.bound * 1.0001 + S.sdf_k + 1e-3; }

// one SDF primitive marched alone (hard union, blend radius 0)
bool t_sdf_single(const Scene &S, const SdfP &q, const Ray &r, double tmin, double tmax, double &tt) {
  double t0;
  const double R = inflated_radius(S, q);
  if (!t_sphere(q.pos, R, r, tmin, tmax, t0)) {
    if ((r.o - q.pos).len2() > R * R) return false;
    t0 = tmin;
  }
  const double il = 1.0 / r.d.len();
  double t = t0;
  for (int i = 0; i < S.sdf_steps; ++i) {
    const double d = sdf_eval1(q, r.at(t));
    if (d < S.sdf_eps) {
      if (t >= tmin && t <= tmax) { tt = t; return true; }
      return false;
    }
    t += d * il;
    if (t > tmax) return false;
  }
  return false;
}

int kind_slot(int type) {
  switch (type) {
    case RB_GEOM_SPHERE: case RB_GEOM_DISPLACED_SPHERE: return 0;
    case RB_GEOM_RECTANGLE: return 1;
    case RB_GEOM_TRIANGLE: return 2;
    default: return 3;
  }
}

bool prim_t(const Scene &S, int i, const Ray &r, double tmin, double tmax, double &t) {
  const Geom &g = S.g[i];
  switch (g.type) {
    case RB_GEOM_SPHERE: case RB_GEOM_DISPLACED_SPHERE: return t_sphere(gv(g, 0), g.p[3], r, tmin, tmax, t);
    case RB_GEOM_RECTANGLE: return t_rect(gv(g, 0), gv(g, 3), gv(g, 6), r, tmin, tmax, t);
    case RB_GEOM_TRIANGLE: return t_tri(gv(g, 0), gv(g, 3), gv(g, 6), r, tmin, tmax, t);
    case RB_GEOM_SDF_PRIMITIVE:
      if (S.sdf_k > 0 || S.sdf_of_geom[i] < 0) return false;  // smooth field handled after traversal
      return t_sdf_single(S, S.sdf[S.sdf_of_geom[i]], r, tmin, tmax, t);
    default: return false;
  }
}

// Smooth-union field of the SDF primitives whose inflated bounding spheres
// overlap [tmin, tmax], folded in index order over those whose window (the
// ray interval inside the inflated sphere) holds the current t; sphere tracing
// on the field's magnitude, each step clamped to the next window entry;
// normal by central differences (step 5e-4) over the hit point's windows;
// material of the nearest primitive.
//
// Convex skip: where one window alone holds t and its primitive is convex
// (sphere, box, rounded box, capsule), the field is that primitive's distance,
// a convex function of t. Once it has grown between two consecutive steps
// (by more than a quarter, so FP32 rounding near the surface cannot fake the
// growth) it keeps growing, so no hit lies before the next window entry: the
// march jumps there, as it would have arrived after enough steps.
bool sdf_convex(int type) {
  return type == RB_SDF_SPHERE || type == RB_SDF_BOX || type == RB_SDF_ROUND_BOX || type == RB_SDF_CAPSULE;
}

bool sdf_field(const Scene &S, const Ray &r, double tmin, double tmax, double &tt, D3 &n, int &mat) {
  struct Win { int idx; double t0, t1; };
  std::vector<Win> c;
  for (int i = 0; i < (int)S.sdf.size(); ++i) {
    const SdfP &q = S.sdf[i];
    const D3 oc = r.o - q.pos;
    const double R = inflated_radius(S, q);
    const double a = dot(r.d, r.d), hb = dot(oc, r.d), cc = dot(oc, oc) - R * R;
    const double disc = hb * hb - a * cc;
    if (disc < 0) continue;
    const double sq = std::sqrt(disc), t0 = (-hb - sq) / a, t1 = (-hb + sq) / a;
    if (t1 >= tmin && t0 <= tmax && c.size() < 24) c.push_back({i, t0, t1});
  }
  if (c.empty()) return false;
  const double FAR = 1e30;
  int held = 0, lone = -1;  // windows holding t at the last evaluation; the last of them
  auto field = [&](const D3 &p, double t, double &next, int *nearest) {
    double F = FAR, best = FAR;
    bool first = true;
    next = FAR;
    held = 0;
    for (const Win &w : c) {
      if (w.t0 > t) { next = std::fmin(next, w.t0); continue; }
      if (t > w.t1) continue;
      ++held;
      lone = w.idx;
      const double d = sdf_eval1(S.sdf[w.idx], p);
      if (nearest && d < best) { best = d; *nearest = w.idx; }
      F = first ? d : smin_poly(F, d, S.sdf_k);
      first = false;
    }
    return F;
  };
  const double il = 1.0 / r.d.len();
  double t = tmin, next, nx;
  double f0 = field(r.at(t), t, next, nullptr);
  for (int k = 0; k < 8 && std::fabs(f0) < 2.0 * S.sdf_eps; ++k) {
    t += 2.0 * S.sdf_eps * il;
    f0 = field(r.at(t), t, next, nullptr);
  }
  const double sgn = f0 < 0 ? -1.0 : 1.0;
  int prev = -1;  // lone convex primitive of the previous step, and its distance there
  double prev_d = 0;
  for (int i = 0; i < S.sdf_steps; ++i) {
    const D3 p = r.at(t);
    const double raw = field(p, t, next, nullptr);
    if (raw == FAR) {
      if (next == FAR || next > tmax) return false;
      t = next;
      prev = -1;
      continue;
    }
    const double F = sgn * raw;
    if (F < S.sdf_eps) {
      if (t > tmax) return false;
      const double e = 5e-4;
      const D3 gr(field(p + D3(e, 0, 0), t, nx, nullptr) - field(p - D3(e, 0, 0), t, nx, nullptr),
                  field(p + D3(0, e, 0), t, nx, nullptr) - field(p - D3(0, e, 0), t, nx, nullptr),
                  field(p + D3(0, 0, e), t, nx, nullptr) - field(p - D3(0, 0, e), t, nx, nullptr));
      const double gl = gr.len();
      n = gl > 0 ? gr / gl : D3(0, 1, 0);
      int nearest = c[0].idx;
      field(p, t, nx, &nearest);
      mat = S.sdf[nearest].mat;
      tt = t;
      return true;
    }
    const int one = (sgn > 0 && held == 1 && sdf_convex(S.sdf[lone].type)) ? lone : -1;
    if (one >= 0 && one == prev && raw > 1.25 * prev_d) {  // convex skip
      if (next == FAR || next > tmax) return false;
      t = next;
      prev = -1;
      continue;
    }
    prev = one;
    prev_d = raw;
    t = std::fmin(t + F * il, next);
    if (t > tmax) return false;
  }
  return false;
}

int trace_bvh(const Scene &S, const Ray &r, double tmin, double tmax, double &tout, bool any, Counters &c);

// Closest (or first) hit: BVH primitives, then the smooth SDF field up to
// the closest primitive hit. A field hit returns -2 with its normal/material.
struct FieldHit {
  D3 n;
  int mat = 0;
};
int trace(const Scene &S, const Ray &r, double tmin, double tmax, double &tout, bool any, Counters &c,
          FieldHit *fh = nullptr) {
  const int h = trace_bvh(S, r, tmin, tmax, tout, any, c);
  if (S.sdf_k > 0 && !S.sdf.empty() && !(any && h >= 0)) {
    double ts;
    D3 n;
    int mat;
    if (sdf_field(S, r, tmin, h >= 0 ? tout : tmax, ts, n, mat)) {
      tout = ts;
      if (fh) { fh->n = n; fh->mat = mat; }
      return -2;
    }
  }
  return h;
}

// hit_scene: DFS with push (far, near) by the ray's sign on the split axis.
int trace_bvh(const Scene &S, const Ray &r, double tmin, double tmax, double &tout, bool any, Counters &c) {
  double closest = tmax;
  int hit = -1;
  if (S.root < 0) {
    for (int i = 0; i < (int)S.g.size(); ++i) {
      double t;
      ++c.prims;
      ++c.kind[kind_slot(S.g[i].type)];
      if (prim_t(S, i, r, tmin, closest, t)) {
        closest = t;
        hit = i;
        if (any) break;
      }
    }
    tout = closest;
    return hit;
  }
  int stack[64];
  int sp = 0;
  stack[sp++] = S.root;
  while (sp > 0) {
    const Node &n = S.n[stack[--sp]];
    ++c.nodes;
    if (!box_hit(r, n.lo, n.hi, tmin, closest)) continue;
    if (n.leaf) {
      for (int i = 0; i < n.b; ++i) {
        double t;
        ++c.prims;
        ++c.kind[kind_slot(S.g[n.a + i].type)];
        if (prim_t(S, n.a + i, r, tmin, closest, t)) {
          closest = t;
          hit = n.a + i;
          if (any) {
            tout = closest;
            return hit;
          }
        }
      }
    } else {
      const double dc = n.axis == 0 ? r.d.x : (n.axis == 1 ? r.d.y : r.d.z);
      const int nearc = dc >= 0 ? n.a : n.b, farc = dc >= 0 ? n.b : n.a;
      if (sp < 32) stack[sp++] = farc;
      if (sp < 32) stack[sp++] = nearc;
    }
  }
  tout = closest;
  return hit;
}

struct Surf {
  D3 p, n, tangent, center;
  bool front, visible;
  int mat;
};

Surf surface(const Scene &S, const Ray &r, int i, double t) {
  const Geom &g = S.g[i];
  Surf s;
  s.visible = g.visible != 0;
  s.mat = g.mat;
  s.p = r.at(t);
  s.center = D3(0, 0, 0);
  if (g.type == RB_GEOM_SPHERE || g.type == RB_GEOM_DISPLACED_SPHERE) {
    const D3 c = gv(g, 0);
    const D3 out = (s.p - c) / g.p[3];
    s.front = dot(r.d, out) < 0;
    s.n = s.front ? out : -out;
    D3 tg = cross(D3(0, 1, 0), out);
    if (tg.len2() < 1e-6) tg = D3(1, 0, 0);
    s.tangent = norm(tg);
    s.center = c;
  } else if (g.type == RB_GEOM_RECTANGLE) {
    const D3 u = gv(g, 3), v = gv(g, 6);
    const D3 n = norm(cross(u, v));
    s.front = dot(r.d, n) < 0;
    s.n = s.front ? n : -n;
    s.tangent = norm(u);
  } else if (g.type == RB_GEOM_SDF_PRIMITIVE) {
    const SdfP &q = S.sdf[S.sdf_of_geom[i]];
    const double e = S.sdf_eps;
    const D3 gr(sdf_eval1(q, s.p + D3(e, 0, 0)) - sdf_eval1(q, s.p - D3(e, 0, 0)),
                sdf_eval1(q, s.p + D3(0, e, 0)) - sdf_eval1(q, s.p - D3(0, e, 0)),
                sdf_eval1(q, s.p + D3(0, 0, e)) - sdf_eval1(q, s.p - D3(0, 0, e)));
    const D3 n = norm(gr);
    s.front = dot(r.d, n) < 0;
    s.n = s.front ? n : -n;
    D3 tg = cross(D3(0, 1, 0), n);
    if (tg.len2() < 1e-6) tg = D3(1, 0, 0);
    s.tangent = norm(tg);
    s.center = q.pos;
  } else {
    const D3 v0 = gv(g, 0), e1 = gv(g, 3) - v0, e2 = gv(g, 6) - v0;
    const D3 geo = norm(cross(e1, e2));
    s.front = dot(r.d, geo) < 0;
    D3 sn = geo;
    if (g.has_normals) {
      const D3 h = cross(r.d, e2);
      const double f = 1.0 / dot(e1, h);
      const D3 sv = r.o - v0;
      const double uu = f * dot(sv, h);
      const double vv = f * dot(r.d, cross(sv, e1));
      sn = norm((1.0 - uu - vv) * gv(g, 9) + uu * gv(g, 12) + vv * gv(g, 15));
      if (dot(sn, geo) < 0) sn = -sn;
    }
    s.n = s.front ? sn : -sn;
    if (g.has_normals && dot(s.n, -r.d) <= 0) s.n = s.front ? geo : -geo;
    s.tangent = norm(e1);
  }
  return s;
}

// --- sampling and materials ------------------------------------------------------
D3 reflect(const D3 &v, const D3 &n) { return v - 2 * dot(v, n) * n; }
D3 refract(const D3 &uv, const D3 &n, double eta) {
  const double ct = std::fmin(dot(-uv, n), 1.0);
  const D3 perp = eta * (uv + ct * n);
  return perp + (-std::sqrt(std::fabs(1.0 - perp.len2()))) * n;
}
double schlick(double c, double ri) {
  double r0 = (1 - ri) / (1 + ri);
  r0 *= r0;
  return r0 + (1 - r0) * std::pow(1 - c, 5);
}
void onb(const D3 &n, D3 &b1, D3 &b2) {  // Duff et al. 2017
  const double sign = std::copysign(1.0, n.z);
  const double a = -1.0 / (sign + n.z);
  const double b = n.x * n.y * a;
  b1 = D3(1.0 + sign * n.x * n.x * a, sign * b, -sign * n.x);
  b2 = D3(b, sign + n.y * n.y * a, -n.y);
}
D3 uniform_sphere(double u1, double u2) {
  const double z = 1 - 2 * u2, r = std::sqrt(std::fmax(0.0, 1 - z * z)), ph = 2 * PI * u1;
  return D3(r * std::cos(ph), r * std::sin(ph), z);
}
D3 cosine_dir(const D3 &n, double u1, double u2, double &cz) {
  D3 b1, b2;
  onb(n, b1, b2);
  const double r = std::sqrt(u1), ph = 2 * PI * u2;
  cz = std::sqrt(std::fmax(0.0, 1 - u1));
  return (r * std::cos(ph)) * b1 + (r * std::sin(ph)) * b2 + cz * n;
}
double ggx_lambda(const D3 &w, double ax, double ay) {
  const double wz2 = w.z * w.z;
  if (wz2 < 1e-16) return 0;
  const double a2 = (ax * w.x) * (ax * w.x) + (ay * w.y) * (ay * w.y);
  return (std::sqrt(1 + a2 / wz2) - 1) * 0.5;
}
D3 ggx_wm(const D3 &wo, double ax, double ay, double u1, double u2) {
  D3 wh = norm(D3(ax * wo.x, ay * wo.y, wo.z));
  if (wh.z < 0) wh = -wh;
  const D3 t1 = wh.z < 0.99999 ? norm(cross(D3(0, 0, 1), wh)) : D3(1, 0, 0);
  const D3 t2 = cross(wh, t1);
  const double r = std::sqrt(u1), ph = 2 * PI * u2;
  const double px = r * std::cos(ph);
  double py = r * std::sin(ph);
  const double h = std::sqrt(std::fmax(0.0, 1 - px * px));
  const double s = (1 + wh.z) * 0.5;
  py = (1 - s) * h + s * py;
  const double pz = std::sqrt(std::fmax(0.0, 1 - px * px - py * py));
  const D3 nh = px * t1 + py * t2 + pz * wh;
  return norm(D3(ax * nh.x, ay * nh.y, std::fmax(1e-6, nh.z)));
}
double fr1(double c2, double s2, double ci, double eta, double k) {
  const double e2 = eta * eta, k2 = k * k, t0 = e2 - k2 - s2;
  const double a2b2 = std::sqrt(std::fmax(t0 * t0 + 4 * e2 * k2, 0.0));
  const double a = std::sqrt(std::fmax((a2b2 + t0) * 0.5, 0.0));
  const double rs = (a2b2 + c2 - 2 * a * ci) / std::fmax(a2b2 + c2 + 2 * a * ci, 1e-10);
  const double rp = rs * (a2b2 * c2 + s2 * s2 - 2 * a * ci * s2) / std::fmax(a2b2 * c2 + s2 * s2 + 2 * a * ci * s2, 1e-10);
  return (rs + rp) * 0.5;
}
D3 fr(double ci, const D3 &eta, const D3 &k) {
  ci = std::fmin(std::fmax(ci, 0.0), 1.0);
  const double c2 = ci * ci, s2 = 1 - c2;
  return D3(fr1(c2, s2, ci, eta.x, k.x), fr1(c2, s2, ci, eta.y, k.y), fr1(c2, s2, ci, eta.z, k.z));
}
D3 fib_point(int i, int n) {
  const double k = i + 0.5, v = k / n, phi = std::acos(1 - 2 * v), th = 2.39996323 * k, s = std::sin(phi);
  return D3(std::cos(th) * s, std::sin(th) * s, std::cos(phi));
}

struct Scat {
  D3 att{1, 1, 1}, emit{0, 0, 0};
  Ray ray;
  double pdf = 0;
  bool scattered = false;
};

Scat scatter(const Globals &G, const Mat &m, const Surf &s, const Ray &in, uint32_t key, int bounce) {
  Scat o;
  D3 color = m.color;
  if (m.pattern) {
    const D3 q = norm(s.p - s.center);
    double best = -1;
    for (int i = 0; i < (int)m.p1; ++i) best = std::fmax(best, dot(q, fib_point(i, (int)m.p1)));
    best = std::fmax(std::fmin(best, 1.0), -1.0);
    const double mask = std::acos(best) < m.p2 ? 0.0 : 1.0;
    color = color * mask + m.pattern_color * (1 - mask);
  }
  const uint32_t d0 = rb_vdim(bounce, RB_SLOT_BSDF);
  auto U = [&](uint32_t d) { return rb_draw_d(key, d); };
  switch (m.kind) {
    case L_LAMB: {
      double cz;
      const D3 w = norm(s.n);
      o.ray.d = cosine_dir(w, U(d0), U(d0 + 1), cz);
      o.ray.o = s.p + 0.0001 * s.n;
      o.att = color;
      o.pdf = cz / PI;
      o.scattered = true;
      break;
    }
    case L_MIRROR: {
      const D3 r = reflect(norm(in.d), s.n);
      o.ray.o = s.p;
      o.ray.d = r;
      o.att = color;
      o.scattered = dot(r, s.n) > 0;
      break;
    }
    case L_ROUGH: {
      const D3 pn = norm(s.n + (m.roughness * G.fuzz) * uniform_sphere(U(d0), U(d0 + 1)));
      const D3 r = reflect(norm(in.d), pn);
      o.ray.o = s.p;
      o.ray.d = r;
      o.att = color;
      o.scattered = dot(r, s.n) > 0;
      break;
    }
    case L_GLASS: {
      const D3 ud = norm(in.d);
      const double ratio = s.front ? 1.0 / G.glass_ior : G.glass_ior;
      const double ct = std::fmin(dot(-ud, s.n), 1.0), st = std::sqrt(1 - ct * ct);
      const bool tir = ratio * st > 1.0;
      const D3 dir = (tir || schlick(ct, ratio) > U(rb_vdim(bounce, RB_SLOT_LOBE))) ? reflect(ud, s.n) : refract(ud, s.n, ratio);
      o.ray.o = s.p;
      o.ray.d = dir;
      o.scattered = true;
      break;
    }
    case L_LIGHT: o.emit = m.emission * G.light; break;
    case L_CONST: o.emit = color; break;
    case L_NORMALS: o.emit = 0.5 * (s.n + D3(1, 1, 1)); break;
    case L_ANISO: {
      const double aspect = std::sqrt(std::fmax(1e-4, 1 - 0.9 * m.anisotropy)), r2 = m.roughness * m.roughness;
      const double ax = std::fmax(1e-4, r2 / aspect), ay = std::fmax(1e-4, r2 * aspect);
      if (std::fmax(ax, ay) < 1e-3) {
        const D3 r = reflect(norm(in.d), s.n);
        o.ray.o = s.p + 0.0001 * s.n;
        o.ray.d = r;
        o.att = color * fr(std::fmax(dot(-norm(in.d), s.n), 0.0), m.eta, m.k);
        o.scattered = dot(r, s.n) > 0;
        break;
      }
      const D3 N = norm(s.n), T = norm(s.tangent - dot(s.tangent, N) * N), B = cross(N, T);
      const D3 wo = norm(-in.d), wol(dot(wo, T), dot(wo, B), dot(wo, N));
      if (wol.z <= 0) break;
      const D3 wm = ggx_wm(wol, ax, ay, U(d0), U(d0 + 1));
      const D3 wil = reflect(-wol, wm);
      if (wil.z <= 0) break;
      const D3 F = fr(std::fmax(dot(wol, wm), 0.0), m.eta, m.k);
      const double g = 1 / (1 + ggx_lambda(wol, ax, ay) + ggx_lambda(wil, ax, ay));
      const double g1 = 1 / (1 + ggx_lambda(wol, ax, ay));
      o.ray.o = s.p + 0.0001 * s.n;
      o.ray.d = wil.x * T + wil.y * B + wil.z * N;
      o.att = color * (F * (g / std::fmax(g1, 1e-6)));
      o.scattered = true;
      break;
    }
    case L_FILM: {
      const D3 ud = norm(in.d);
      const double ci = std::fmax(std::fabs(dot(-ud, s.n)), 0.001), n0 = m.ior, n1 = m.film_ior, d = m.film_thickness;
      const double si = std::sqrt(std::fmax(0.0, 1 - ci * ci)), stt = (n0 / n1) * si;
      const double ctt = stt >= 1 ? 0.0 : std::sqrt(1 - stt * stt);
      double r01 = (n0 - n1) / (n0 + n1);
      r01 *= r01;
      const double R01 = r01 + (1 - r01) * std::pow(1 - ci, 5);
      double r12 = (n1 - n0) / (n1 + n0);
      r12 *= r12;
      const double R12 = r12 + (1 - r12) * std::pow(1 - ctt, 5);
      const double sq = std::sqrt(R01 * R12);
      double Rc[3];
      const double lam[3] = {650, 550, 450};
      for (int i = 0; i < 3; ++i) {
        const double c = std::cos((4 * PI * n1 * d * ctt) / lam[i]);
        Rc[i] = (R01 + R12 + 2 * sq * c) / std::fmax(1 + R01 * R12 + 2 * sq * c, 1e-8);
      }
      const double avg = (Rc[0] + Rc[1] + Rc[2]) / 3;
      if (U(rb_vdim(bounce, RB_SLOT_LOBE)) < avg) {
        const D3 r = reflect(ud, s.n);
        o.ray.o = s.p + 0.0001 * s.n;
        o.ray.d = r;
        o.att = D3(Rc[0], Rc[1], Rc[2]) * (1 / std::fmax(avg, 0.001));
        o.scattered = dot(r, s.n) > 0;
      } else {
        o.ray.o = s.p - 0.0001 * s.n;
        o.ray.d = ud;
        o.att = D3(1 - Rc[0], 1 - Rc[1], 1 - Rc[2]) * (1 / std::fmax(1 - avg, 0.001));
        o.scattered = true;
      }
      break;
    }
    case L_COAT: {
      const D3 ud = norm(in.d);
      const double F = schlick(std::fmin(dot(-ud, s.n), 1.0), m.ior);
      if (U(rb_vdim(bounce, RB_SLOT_LOBE)) < F) {
        const uint32_t d3 = rb_vdim(bounce, RB_SLOT_BSDF2);
        const D3 pn = m.roughness > 1e-3 ? norm(s.n + m.roughness * uniform_sphere(U(d3), U(d3 + 1))) : s.n;
        const D3 r = reflect(ud, pn);
        o.ray.o = s.p + 0.0001 * s.n;
        o.ray.d = r;
        o.scattered = dot(r, s.n) > 0;
      } else {
        double cz;
        o.ray.o = s.p + 0.0001 * s.n;
        o.ray.d = cosine_dir(norm(s.n), U(d0), U(d0 + 1), cz);
        o.att = color;
        o.scattered = true;
      }
      break;
    }
    default: break;
  }
  return o;
}

double mis2(double a, double b) { return a * a / (a * a + b * b); }

bool sample_light(const Scene &S, const Globals &G, double ul, double u1, double u2, D3 &p, D3 &n, D3 &Le) {
  if (S.lights.empty()) return false;
  const double target = ul * S.light_area;
  size_t i = 0;
  while (i + 1 < S.lights.size() && S.lights[i].cdf <= target) ++i;
  const Geom &g = S.g[S.lights[i].prim];
  if (g.type == RB_GEOM_RECTANGLE) {
    p = gv(g, 0) + u1 * gv(g, 3) + u2 * gv(g, 6);
    n = norm(cross(gv(g, 3), gv(g, 6)));
  } else if (g.type == RB_GEOM_TRIANGLE) {
    const D3 e1 = gv(g, 3) - gv(g, 0), e2 = gv(g, 6) - gv(g, 0);
    const double su = std::sqrt(u1);
    p = gv(g, 0) + (su * (1 - u2)) * e1 + (su * u2) * e2;
    n = norm(cross(e1, e2));
  } else {
    const D3 d = uniform_sphere(u1, u2);
    p = gv(g, 0) + g.p[3] * d;
    n = d;
  }
  Le = S.m[g.mat].emission * G.light;
  return true;
}

D3 sky(const D3 &d) {
  const D3 u = norm(d);
  const double t = 0.5 * (u.y + 1.0);
  return (1.0 - t) * D3(1, 1, 1) + t * D3(0.5, 0.7, 1.0);
}

// One path of one sample (ray_color, cuda_raytracer.cuh:858-933).
D3 radiance(const Scene &S, const Globals &G, Ray ray, uint32_t key, int depth, Counters &c) {
  D3 L(0, 0, 0), thr(1, 1, 1);
  double prev_pdf = 0;
  for (int bounce = 0; bounce < depth; ++bounce) {
    ++c.segments;
    double t;
    FieldHit fh;
    const int h = trace(S, ray, 0.001, 3.4028234663852886e38, t, false, c, &fh);
    if (h == -1) {
      L = L + thr * sky(ray.d) * G.background;
      return L;
    }
    Surf s;
    if (h == -2) {
      s.p = ray.at(t) + (4.0 * S.sdf_eps) * fh.n * (dot(ray.d, fh.n) < 0 ? 1.0 : -1.0);
      s.front = dot(ray.d, fh.n) < 0;
      s.n = s.front ? fh.n : -fh.n;
      D3 tg = cross(D3(0, 1, 0), fh.n);
      if (tg.len2() < 1e-6) tg = D3(1, 0, 0);
      s.tangent = norm(tg);
      s.center = D3(0, 0, 0);
      s.visible = true;
      s.mat = fh.mat;
    } else {
      s = surface(S, ray, h, t);
    }
    if (!s.visible && bounce == 0) {
      ray.o = s.p + ray.d * 0.01;
      continue;
    }
    if (s.mat < 0 || s.mat >= (int)S.m.size()) return L;
    const Mat &m = S.m[s.mat];
    ++c.shade[m.kind == L_LAMB ? 0 : (m.kind == L_MIRROR || m.kind == L_ROUGH) ? 1 : m.kind == L_GLASS ? 2
              : (m.kind == L_LIGHT || m.kind == L_CONST || m.kind == L_NORMALS) ? 3 : 4];
    const Scat o = scatter(G, m, s, ray, key, bounce);
    if (o.emit.len2() > 0) {
      double w = 1;
      if (G.nee && prev_pdf > 0 && m.kind == L_LIGHT && !S.lights.empty()) {
        const double dl = t * ray.d.len();
        const double cl = std::fabs(dot(s.n, norm(ray.d)));
        const double pl = cl > 0 ? dl * dl / (cl * S.light_area) : 0;
        w = mis2(prev_pdf, pl);
      }
      L = L + thr * o.emit * w;
    }
    if (!o.scattered) return L;
    if (G.nee) {
      prev_pdf = 0;
      if (m.kind == L_LAMB && bounce + 1 < depth && !S.lights.empty()) {
        const uint32_t dl = rb_vdim(bounce, RB_SLOT_LIGHT);
        D3 lp, ln, Le;
        if (sample_light(S, G, rb_draw_d(key, dl), rb_draw_d(key, dl + 1), rb_draw_d(key, dl + 2), lp, ln, Le)) {
          const D3 dv = lp - o.ray.o;
          const double d2 = dv.len2(), dist = std::sqrt(d2);
          const D3 wi = dv / dist;
          const double cs = dot(norm(s.n), wi), cl = std::fabs(dot(ln, wi));
          if (cs > 0 && cl > 0) {
            ++c.shadow;
            double ts;
            Ray sr{o.ray.o, wi};
            if (trace(S, sr, 0.001, dist * (1 - 1e-4), ts, true, c) == -1) {
              const double pl = d2 / (cl * S.light_area), pb = cs / PI;
              L = L + thr * o.att * Le * (cs / PI * mis2(pl, pb) / pl);
            }
          }
        }
        prev_pdf = o.pdf;
      }
    }
    thr = thr * o.att;
    if (bounce > 0) {
      const double sp = std::fmin(std::fmax(thr.x, std::fmax(thr.y, thr.z)), 0.95);
      if (rb_draw_d(key, rb_vdim(bounce, RB_SLOT_RR)) > sp) return L;
      thr = thr / sp;
    }
    ray = o.ray;
  }
  return L;
}

Ray camera_ray(const double *fr, const Globals &G, int x, int y, uint32_t key) {
  const D3 center(fr[0], fr[1], fr[2]), p00(fr[3], fr[4], fr[5]), du(fr[6], fr[7], fr[8]), dv(fr[9], fr[10], fr[11]);
  const D3 cu(fr[12], fr[13], fr[14]), cv(fr[15], fr[16], fr[17]);
  const double ou = rb_draw_d(key, RB_DIM_JITTER) - 0.5, ov = rb_draw_d(key, RB_DIM_JITTER + 1) - 0.5;
  Ray r;
  r.o = center;
  r.d = (p00 + (x + ou) * du + (y + ov) * dv) - center;
  if (G.dof && G.aperture > 0) {
    const D3 focus = center + G.focus * norm(r.d);
    const double rr = std::sqrt(rb_draw_d(key, RB_DIM_LENS)), ph = 2 * PI * rb_draw_d(key, RB_DIM_LENS + 1);
    r.o = center + G.aperture * ((rr * std::cos(ph)) * cu + (rr * std::sin(ph)) * cv);
    r.d = focus - r.o;
  }
  return r;
}

}  // namespace

extern "C" {

struct orc_globals {
  double light, background, fuzz, glass_ior;
  int dof;
  double aperture, focus;
  int nee;
};

// geoms: n x 32 rows as rb_scene_export_geometry_full (leaf order); nodes in
// the reference layout (pre-order, leaves included); root < 0: linear scan.
void *orc_scene_create(const double *geoms, int64_t n, const rb_material_desc *mats, int nmat,
                       const double *bounds, const int32_t *a, const int32_t *b, const uint8_t *leaf,
                       const uint8_t *axis, int64_t nnodes, int root) {
  Scene *S = new Scene();
  S->g.resize(n);
  for (int64_t i = 0; i < n; ++i) {
    const double *r = geoms + 32 * i;
    Geom &g = S->g[i];
    g.type = (int)r[0];
    g.mat = (int)r[1];
    g.visible = (int)r[2];
    g.has_normals = (int)r[3];
    for (int k = 0; k < 18; ++k) g.p[k] = r[4 + k];
  }
  for (int i = 0; i < nmat; ++i) S->m.push_back(resolve(mats[i]));
  S->n.resize(nnodes);
  for (int64_t i = 0; i < nnodes; ++i) {
    Node &nd = S->n[i];
    for (int k = 0; k < 3; ++k) { nd.lo[k] = bounds[6 * i + k]; nd.hi[k] = bounds[6 * i + 3 + k]; }
    nd.a = a[i];
    nd.b = b[i];
    nd.leaf = leaf[i];
    nd.axis = axis[i];
  }
  S->root = nnodes > 0 ? root : -1;
  S->sdf_of_geom.assign(n, -1);
  for (int64_t i = 0; i < n; ++i) {
    const Geom &g = S->g[i];
    if (g.type != RB_GEOM_SDF_PRIMITIVE) continue;
    const int t = (int)g.p[0];
    if (t != RB_SDF_SPHERE && t != RB_SDF_BOX && t != RB_SDF_ROUND_BOX && t != RB_SDF_TORUS && t != RB_SDF_CAPSULE)
      continue;
    SdfP q;
    q.type = t;
    q.mat = g.mat;
    q.pos = gv(g, 1);
    q.a = g.p[4]; q.b = g.p[5]; q.c = g.p[6];
    q.round = t == RB_SDF_ROUND_BOX ? 0.2 * std::fmin(g.p[4], std::fmin(g.p[5], g.p[6])) : 0.0;
    const double a = std::fabs(q.a), b = std::fabs(q.b), c = std::fabs(q.c);
    q.bound = (t == RB_SDF_SPHERE) ? a : (t == RB_SDF_TORUS) ? a + b : (t == RB_SDF_CAPSULE) ? a + 0.5 * b
                                                                                               : std::sqrt(a * a + b * b + c * c);
    const double cx = std::cos(g.p[7]), sx = std::sin(g.p[7]), cy = std::cos(g.p[8]), sy = std::sin(g.p[8]);
    const double cz = std::cos(g.p[9]), sz = std::sin(g.p[9]);
    const double R[3][3] = {{cz * cy, cz * sy * sx - sz * cx, cz * sy * cx + sz * sx},
                            {sz * cy, sz * sy * sx + cz * cx, sz * sy * cx - cz * sx},
                            {-sy, cy * sx, cy * cx}};
    for (int a2 = 0; a2 < 3; ++a2)
      for (int b2 = 0; b2 < 3; ++b2) q.R[3 * a2 + b2] = R[b2][a2];
    S->sdf_of_geom[i] = (int)S->sdf.size();
    S->sdf.push_back(q);
  }
  for (int64_t i = 0; i < n; ++i) {
    const Geom &g = S->g[i];
    if (g.mat < 0 || g.mat >= nmat || S->m[g.mat].kind != L_LIGHT) continue;
    const Mat &m = S->m[g.mat];
    if (!(m.emission.x > 0 || m.emission.y > 0 || m.emission.z > 0)) continue;
    double area = 0;
    if (g.type == RB_GEOM_RECTANGLE) area = cross(gv(g, 3), gv(g, 6)).len();
    else if (g.type == RB_GEOM_TRIANGLE) area = 0.5 * cross(gv(g, 3) - gv(g, 0), gv(g, 6) - gv(g, 0)).len();
    else if (g.type == RB_GEOM_SPHERE) area = 4 * PI * g.p[3] * g.p[3];
    if (area <= 0) continue;
    S->light_area += area;
    S->lights.push_back({(int)i, area, S->light_area});
  }
  return S;
}

void orc_scene_destroy(void *s) { delete static_cast<Scene *>(s); }

// Smooth-union radius, step limit and hit epsilon of the SDF primitives.
void orc_scene_set_sdf(void *sp, double k, int steps, double eps) {
  Scene &S = *static_cast<Scene *>(sp);
  S.sdf_k = k;
  S.sdf_steps = steps;
  S.sdf_eps = eps;
}

// Pixel-centre primary hits; counters[0..1] += nodes visited, prims tested.
void orc_primary(void *sp, int w, int h, const double *fr, int32_t *ids, double *tout, int64_t *counters, int threads) {
  const Scene &S = *static_cast<Scene *>(sp);
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int64_t> nodes{0}, prims{0};
  auto work = [&](int t) {
    Counters c;
    for (int y = t; y < h; y += threads)
      for (int x = 0; x < w; ++x) {
        const D3 center(fr[0], fr[1], fr[2]), p00(fr[3], fr[4], fr[5]), du(fr[6], fr[7], fr[8]), dv(fr[9], fr[10], fr[11]);
        Ray r{center, (p00 + (double)x * du + (double)y * dv) - center};
        double t;
        const int id = trace(S, r, 0.001, 3.4028234663852886e38, t, false, c);
        ids[y * w + x] = id;
        if (tout) tout[y * w + x] = id != -1 ? t : -1.0;  // smooth-field hits (-2) report t too
      }
    nodes += c.nodes;
    prims += c.prims;
  };
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t) th.emplace_back(work, t);
  for (auto &t : th) t.join();
  if (counters) {
    counters[0] += nodes.load();
    counters[1] += prims.load();
  }
}

// Renders samples [sample_base, sample_base + spp) for the listed pixels
// (pixel indices y * w + x; NULL = all w*h) and writes per-pixel radiance SUMS
// (FP64) to out (npix x 3). counters (ORC_NCOUNTERS): nodes, prims, segments,
// paths, shadow rays, primitive tests by kind (sphere, rectangle, triangle,
// SDF), shading events by class (Lambert, mirror, glass, emitter, GGX/film/coat).
void orc_render(void *sp, int w, int h, const double *fr, const int32_t *pixels, int npix, int spp, int sample_base,
                int depth, const orc_globals *g, uint32_t seed, uint32_t salt, double *out, int threads,
                int64_t *counters) {
  const Scene &S = *static_cast<Scene *>(sp);
  Globals G{g->light, g->background, g->fuzz, g->glass_ior, g->dof, g->aperture, g->focus, g->nee};
  const int n = pixels ? npix : w * h;
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int> next{0};
  std::vector<Counters> cs(threads);
  auto work = [&](int t) {
    Counters &c = cs[t];
    while (true) {
      const int i0 = next.fetch_add(64);
      if (i0 >= n) break;
      for (int i = i0; i < std::min(n, i0 + 64); ++i) {
        const int pix = pixels ? pixels[i] : i;
        const int x = pix % w, y = pix / w;
        D3 sum(0, 0, 0);
        for (int s = 0; s < spp; ++s) {
          const uint32_t key = rb_path_key(seed, salt, (uint32_t)pix, (uint32_t)(sample_base + s));
          ++c.paths;
          sum = sum + radiance(S, G, camera_ray(fr, G, x, y, key), key, depth, c);
        }
        out[3 * i] = sum.x;
        out[3 * i + 1] = sum.y;
        out[3 * i + 2] = sum.z;
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t) th.emplace_back(work, t);
  for (auto &t : th) t.join();
  if (counters)
    for (auto &c : cs) {
      counters[0] += c.nodes;
      counters[1] += c.prims;
      counters[2] += c.segments;
      counters[3] += c.paths;
      counters[4] += c.shadow;
      for (int k = 0; k < 4; ++k) counters[5 + k] += c.kind[k];
      for (int k = 0; k < 5; ++k) counters[9 + k] += c.shade[k];
    }
}

}  // extern "C"
