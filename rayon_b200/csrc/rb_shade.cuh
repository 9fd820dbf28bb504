// Material scatter, next-event estimation helpers, golf-ball surface and SDF
// marching for the B200 render path.
//
// Scatter semantics per legacy material follow scatter_material
// (src/rayon/gpu_renderers/cuda_raytracer.cuh:613-850), including the
// reference's quirks: METAL/ROUGH_MIRROR roughness defaults to 0.3 and is
// scaled by the global metal fuzziness; GLASS uses the global IOR and feeds
// the refraction ratio to Schlick; lights emit on both faces and end the
// path. Sampling routines are this project's own where the distribution is
// the same: a branch-free orthonormal basis (Duff et al. 2017, "Building an
// Orthonormal Basis, Revisited") and the closed-form uniform sphere mapping
// z = 1 - 2u (equal to acos-based polar sampling).
#pragma once

#include "rb_device.cuh"

namespace rbd {

#define RB_PI 3.14159265358979323846f

__device__ __forceinline__ f3 reflect(const f3 &v, const f3 &n) { return v - 2 * dot(v, n) * n; }

__device__ __forceinline__ f3 refract(const f3 &uv, const f3 &n, float eta) {
  float cos_theta = fminf(dot(-uv, n), 1.0f);
  f3 perp = eta * (uv + cos_theta * n);
  f3 par = -sqrtf(fabsf(1.0f - perp.length_squared())) * n;
  return perp + par;
}

__device__ __forceinline__ float schlick(float cosine, float ref_idx) {
  float r0 = (1 - ref_idx) / (1 + ref_idx);
  r0 = r0 * r0;
  const float m = 1 - cosine;
  const float m2 = m * m;
  return r0 + (1 - r0) * (m2 * m2 * m);
}

__device__ __forceinline__ void onb(const f3 &n, f3 &b1, f3 &b2) {
  const float sign = copysignf(1.0f, n.z);
  const float a = -1.0f / (sign + n.z);
  const float b = n.x * n.y * a;
  b1 = f3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
  b2 = f3(b, sign + n.y * n.y * a, -n.y);
}

__device__ __forceinline__ f3 uniform_sphere(float u1, float u2) {
  const float z = 1.0f - 2.0f * u2;
  const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  float s, c;
  __sincosf(2.0f * RB_PI * u1, &s, &c);
  return f3(r * c, r * s, z);
}

// Cosine-weighted direction about n; pdf = cos / pi.
__device__ __forceinline__ f3 cosine_dir(const f3 &n, float u1, float u2, float &cos_out) {
  f3 b1, b2;
  onb(n, b1, b2);
  const float r = sqrtf(u1);
  float s, c;
  __sincosf(2.0f * RB_PI * u2, &s, &c);
  const float z = sqrtf(fmaxf(0.0f, 1.0f - u1));
  cos_out = z;
  return (r * c) * b1 + (r * s) * b2 + z * n;
}

// ---------------------------------------------------------------------------
// GGX microfacet (Smith masking, VNDF sampling, conductor Fresnel) as in
// microfacet_ggx.cuh:21-111 (PBR Book 4th ed. 9.6)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float ggx_lambda(const f3 &w, float ax, float ay) {
  const float wz2 = w.z * w.z;
  if (wz2 < 1e-16f) return 0.0f;
  const float a2 = (ax * w.x) * (ax * w.x) + (ay * w.y) * (ay * w.y);
  return (sqrtf(1.0f + a2 / wz2) - 1.0f) * 0.5f;
}
__device__ __forceinline__ float ggx_g1(const f3 &w, float ax, float ay) { return 1.0f / (1.0f + ggx_lambda(w, ax, ay)); }
__device__ __forceinline__ float ggx_g(const f3 &wo, const f3 &wi, float ax, float ay) {
  return 1.0f / (1.0f + ggx_lambda(wo, ax, ay) + ggx_lambda(wi, ax, ay));
}
__device__ __forceinline__ f3 ggx_sample_wm(const f3 &wo, float ax, float ay, float u1, float u2) {
  f3 wh = normalize(f3(ax * wo.x, ay * wo.y, wo.z));
  if (wh.z < 0.0f) wh = -wh;
  const f3 t1 = (wh.z < 0.99999f) ? normalize(cross(f3(0.0f, 0.0f, 1.0f), wh)) : f3(1.0f, 0.0f, 0.0f);
  const f3 t2 = cross(wh, t1);
  const float r = sqrtf(u1);
  float sp, cp;
  __sincosf(2.0f * RB_PI * u2, &sp, &cp);
  const float px = r * cp;
  float py = r * sp;
  const float h = sqrtf(fmaxf(0.0f, 1.0f - px * px));
  const float s = (1.0f + wh.z) * 0.5f;
  py = (1.0f - s) * h + s * py;
  const float pz = sqrtf(fmaxf(0.0f, 1.0f - px * px - py * py));
  const f3 nh = px * t1 + py * t2 + pz * wh;
  return normalize(f3(ax * nh.x, ay * nh.y, fmaxf(1e-6f, nh.z)));
}
__device__ __forceinline__ float fr_conductor1(float cos2, float sin2, float ci, float eta, float k) {
  const float eta2 = eta * eta, k2 = k * k;
  const float t0 = eta2 - k2 - sin2;
  const float a2b2 = sqrtf(fmaxf(t0 * t0 + 4.0f * eta2 * k2, 0.0f));
  const float a = sqrtf(fmaxf((a2b2 + t0) * 0.5f, 0.0f));
  const float rs = (a2b2 + cos2 - 2.0f * a * ci) / fmaxf(a2b2 + cos2 + 2.0f * a * ci, 1e-10f);
  const float rp_n = a2b2 * cos2 + sin2 * sin2 - 2.0f * a * ci * sin2;
  const float rp_d = a2b2 * cos2 + sin2 * sin2 + 2.0f * a * ci * sin2;
  const float rp = rs * rp_n / fmaxf(rp_d, 1e-10f);
  return (rs + rp) * 0.5f;
}
__device__ __forceinline__ f3 fr_conductor(float ci, const f3 &eta, const f3 &k) {
  ci = fminf(fmaxf(ci, 0.0f), 1.0f);
  const float c2 = ci * ci, s2 = 1.0f - c2;
  return f3(fr_conductor1(c2, s2, ci, eta.x, k.x), fr_conductor1(c2, s2, ci, eta.y, k.y),
            fr_conductor1(c2, s2, ci, eta.z, k.z));
}

// ---------------------------------------------------------------------------
// Procedural Fibonacci-dot pattern (cuda_raytracer.cuh:377-416)
// ---------------------------------------------------------------------------
__device__ __forceinline__ f3 fib_point(int i, int n) {
  const float ga = 2.39996323f;  // golden angle
  const float k = (float)i + 0.5f;
  const float v = k / (float)n;
  const float phi = acosf(1.0f - 2.0f * v);
  const float theta = ga * k;
  const float s = sinf(phi);
  return f3(cosf(theta) * s, sinf(theta) * s, cosf(phi));
}
static __device__ __noinline__ f3 fib_dots(const DevMaterial &m, const f3 &base, const f3 &p, const f3 &c) {
  const f3 q = normalize(normalize(p - c));
  const int n = min(max((int)m.pattern_p1, 0), 4096);
  float best = -1.0f;
  for (int i = 0; i < n; ++i) best = fmaxf(best, dot(q, fib_point(i, n)));
  best = fmaxf(fminf(best, 1.0f), -1.0f);
  const float mask = acosf(best) < m.pattern_p2 ? 0.0f : 1.0f;
  return base * mask + m.pattern_color * (1.0f - mask);
}

// ---------------------------------------------------------------------------
// Scatter
// ---------------------------------------------------------------------------
struct ScatterOut {
  f3 att;        // throughput factor
  f3 emit;       // emitted radiance (before throughput)
  Ray ray;       // continuation
  float pdf;     // solid-angle pdf of a diffuse (Lambert) sample, 0 otherwise
  bool scattered;
};

// Material classes a kernel is specialised for (the host picks the smallest
// class covering a scene's materials and primitive kinds):
//   RB_MS_DIFFUSE  Lambert, light, constant, normals
//   RB_MS_CLASSIC  + mirror, rough mirror, glass
//   RB_MS_FULL     + GGX conductor, thin film, clear coat, patterns,
//                  displaced spheres
//   RB_MS_SDF      + SDF primitives (hard union and the smooth-union field)
#define RB_MS_DIFFUSE 1
#define RB_MS_CLASSIC 2
#define RB_MS_FULL 3
#define RB_MS_SDF 4

template <int MS>
__device__ __forceinline__ ScatterOut scatter(const Globals &G, const DevMaterial &m, const Surface &s, const Ray &in,
                                              uint32_t key, int bounce) {
  ScatterOut o;
  o.emit = f3(0.0f, 0.0f, 0.0f);
  o.att = f3(1.0f, 1.0f, 1.0f);
  o.pdf = 0.0f;
  o.scattered = false;
  f3 color = m.color;
  if (MS >= RB_MS_FULL && m.pattern == 1) color = fib_dots(m, color, s.p, s.center);
  const uint32_t d0 = rb_vdim(bounce, RB_SLOT_BSDF);
  switch (m.kind) {
    case L_LAMBERTIAN: {
      const f3 w = normalize(s.n);
      float cz;
      const f3 dir = cosine_dir(w, rb_draw(key, d0), rb_draw(key, d0 + 1), cz);
      o.ray.o = s.p + 0.0001f * s.n;
      o.ray.d = dir;
      o.att = color;
      o.pdf = cz * (1.0f / RB_PI);
      o.scattered = true;
      break;
    }
    case L_MIRROR: {
      if (MS < RB_MS_CLASSIC) break;
      const f3 r = reflect(normalize(in.d), s.n);
      o.ray.o = s.p;
      o.ray.d = r;
      o.att = color;
      o.scattered = dot(r, s.n) > 0.0f;
      break;
    }
    case L_ROUGH_MIRROR: {
      if (MS < RB_MS_CLASSIC) break;
      const f3 pn = normalize(s.n + (m.roughness * G.metal_fuzziness) * uniform_sphere(rb_draw(key, d0), rb_draw(key, d0 + 1)));
      const f3 r = reflect(normalize(in.d), pn);
      o.ray.o = s.p;
      o.ray.d = r;
      o.att = color;
      o.scattered = dot(r, s.n) > 0.0f;
      break;
    }
    case L_GLASS: {
      if (MS < RB_MS_CLASSIC) break;
      const f3 ud = normalize(in.d);
      const float ri = G.glass_ior;
      const float ratio = s.front ? (1.0f / ri) : ri;
      const float ct = fminf(dot(-ud, s.n), 1.0f);
      const float st = sqrtf(1.0f - ct * ct);
      const bool tir = ratio * st > 1.0f;
      f3 dir;
      if (tir || schlick(ct, ratio) > rb_draw(key, rb_vdim(bounce, RB_SLOT_LOBE)))
        dir = reflect(ud, s.n);
      else
        dir = refract(ud, s.n, ratio);
      o.ray.o = s.p;
      o.ray.d = dir;
      o.scattered = true;
      break;
    }
    case L_LIGHT:
      o.emit = m.emission * G.light_intensity;
      break;
    case L_CONSTANT:
      o.emit = color;
      break;
    case L_SHOW_NORMALS:
      o.emit = 0.5f * (s.n + f3(1.0f, 1.0f, 1.0f));
      break;
    case L_ANISO_METAL: {
      if (MS < RB_MS_FULL) break;
      const float aspect = sqrtf(fmaxf(1e-4f, 1.0f - 0.9f * m.anisotropy));
      const float r2 = m.roughness * m.roughness;
      const float ax = fmaxf(1e-4f, r2 / aspect), ay = fmaxf(1e-4f, r2 * aspect);
      if (fmaxf(ax, ay) < 1e-3f) {
        const f3 r = reflect(normalize(in.d), s.n);
        o.ray.o = s.p + 0.0001f * s.n;
        o.ray.d = r;
        const float ci = fmaxf(dot(-normalize(in.d), s.n), 0.0f);
        o.att = color * fr_conductor(ci, m.eta, m.k);
        o.scattered = dot(r, s.n) > 0.0f;
        break;
      }
      const f3 N = normalize(s.n);
      const f3 T = normalize(s.tangent - dot(s.tangent, N) * N);
      const f3 B = cross(N, T);
      const f3 wo = normalize(-in.d);
      const f3 wol(dot(wo, T), dot(wo, B), dot(wo, N));
      if (wol.z <= 0.0f) break;
      const f3 wm = ggx_sample_wm(wol, ax, ay, rb_draw(key, d0), rb_draw(key, d0 + 1));
      const f3 wil = reflect(-wol, wm);
      if (wil.z <= 0.0f) break;
      const f3 wiw = wil.x * T + wil.y * B + wil.z * N;
      const f3 F = fr_conductor(fmaxf(dot(wol, wm), 0.0f), m.eta, m.k);
      const float g = ggx_g(wol, wil, ax, ay), g1 = ggx_g1(wol, ax, ay);
      o.ray.o = s.p + 0.0001f * s.n;
      o.ray.d = wiw;
      o.att = color * (F * (g / fmaxf(g1, 1e-6f)));
      o.scattered = true;
      break;
    }
    case L_THIN_FILM: {
      if (MS < RB_MS_FULL) break;
      const f3 ud = normalize(in.d);
      const float ci = fmaxf(fabsf(dot(-ud, s.n)), 0.001f);
      const float n0 = m.ior, n1 = m.film_ior, dd = m.film_thickness;
      const float si = sqrtf(fmaxf(0.0f, 1.0f - ci * ci));
      const float stt = (n0 / n1) * si;
      const float ctt = (stt >= 1.0f) ? 0.0f : sqrtf(1.0f - stt * stt);
      float r01 = (n0 - n1) / (n0 + n1);
      r01 *= r01;
      const float x01 = 1.0f - ci;
      const float R01 = r01 + (1.0f - r01) * x01 * x01 * x01 * x01 * x01;
      float r12 = (n1 - n0) / (n1 + n0);
      r12 *= r12;
      const float x12 = 1.0f - ctt;
      const float R12 = r12 + (1.0f - r12) * x12 * x12 * x12 * x12 * x12;
      const float sq = sqrtf(R01 * R12);
      float Rc[3];
      const float lam[3] = {650.0f, 550.0f, 450.0f};
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const float delta = (4.0f * RB_PI * n1 * dd * ctt) / lam[i];
        const float cd = __cosf(delta);
        Rc[i] = (R01 + R12 + 2.0f * sq * cd) / fmaxf(1.0f + R01 * R12 + 2.0f * sq * cd, 1e-8f);
      }
      const float avg = (Rc[0] + Rc[1] + Rc[2]) / 3.0f;
      if (rb_draw(key, rb_vdim(bounce, RB_SLOT_LOBE)) < avg) {
        const f3 r = reflect(ud, s.n);
        o.ray.o = s.p + 0.0001f * s.n;
        o.ray.d = r;
        o.att = f3(Rc[0], Rc[1], Rc[2]) * (1.0f / fmaxf(avg, 0.001f));
        o.scattered = dot(r, s.n) > 0.0f;
      } else {
        o.ray.o = s.p - 0.0001f * s.n;
        o.ray.d = ud;
        o.att = f3(1.0f - Rc[0], 1.0f - Rc[1], 1.0f - Rc[2]) * (1.0f / fmaxf(1.0f - avg, 0.001f));
        o.scattered = true;
      }
      break;
    }
    case L_CLEAR_COAT: {
      if (MS < RB_MS_FULL) break;
      const f3 ud = normalize(in.d);
      const float ct = fminf(dot(-ud, s.n), 1.0f);
      const float F = schlick(ct, m.ior);
      if (rb_draw(key, rb_vdim(bounce, RB_SLOT_LOBE)) < F) {
        const uint32_t d3 = rb_vdim(bounce, RB_SLOT_BSDF2);
        const f3 pn = (m.roughness > 1e-3f)
                          ? normalize(s.n + m.roughness * uniform_sphere(rb_draw(key, d3), rb_draw(key, d3 + 1)))
                          : s.n;
        const f3 r = reflect(ud, pn);
        o.ray.o = s.p + 0.0001f * s.n;
        o.ray.d = r;
        o.scattered = dot(r, s.n) > 0.0f;
      } else {
        const f3 w = normalize(s.n);
        float cz;
        o.ray.o = s.p + 0.0001f * s.n;
        o.ray.d = cosine_dir(w, rb_draw(key, d0), rb_draw(key, d0 + 1), cz);
        o.att = color;
        o.scattered = true;
      }
      break;
    }
    default:
      break;  // absorbed
  }
  return o;
}

// Sky gradient (cuda_raytracer.cuh:924-929).
__device__ __forceinline__ f3 sky(const f3 &d) {
  const f3 u = normalize(d);
  const float t = 0.5f * (u.y + 1.0f);
  return (1.0f - t) * f3(1.0f, 1.0f, 1.0f) + t * f3(0.5f, 0.7f, 1.0f);
}

// ---------------------------------------------------------------------------
// Next-event estimation on area lights (new on the GPU path)
// ---------------------------------------------------------------------------
// Light choice proportional to area, then a uniform point on the chosen
// emitter: area pdf = 1 / total area for every point of every emitter.
struct LightSample {
  f3 p, n, Le;
};

__device__ __forceinline__ bool sample_light(const SceneView &S, const Globals &G, float ul, float u1, float u2,
                                             LightSample &ls) {
  if (S.num_lights <= 0) return false;
  const float target = ul * S.light_area;
  int lo = 0, hi = S.num_lights - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (S.lights[mid].cdf <= target) lo = mid + 1;
    else hi = mid;
  }
  const int prim = S.lights[lo].prim;
  const float4 *pr = S.prims + 3 * (size_t)prim;
  const float4 a = __ldg(pr), b = __ldg(pr + 1), c = __ldg(pr + 2);
  const uint32_t tag = __float_as_uint(c.w);
  const uint32_t kind = tag_kind(tag);
  if (kind == PK_RECT) {
    const f3 u(a.w, b.x, b.y), v(b.z, b.w, c.x);
    ls.p = f3(a.x, a.y, a.z) + u1 * u + u2 * v;
    ls.n = normalize(cross(u, v));
  } else if (kind == PK_TRI) {
    const f3 e1(a.w, b.x, b.y), e2(b.z, b.w, c.x);
    const float su = sqrtf(u1);
    ls.p = f3(a.x, a.y, a.z) + (su * (1.0f - u2)) * e1 + (su * u2) * e2;
    ls.n = normalize(cross(e1, e2));
  } else {  // sphere
    const f3 d = uniform_sphere(u1, u2);
    ls.p = f3(a.x, a.y, a.z) + a.w * d;
    ls.n = d;
  }
  ls.Le = S.mats[tag_material(tag)].emission * G.light_intensity;
  return true;
}

// Power-heuristic weight of strategy a against b.
__device__ __forceinline__ float mis2(float a, float b) {
  const float a2 = a * a, b2 = b * b;
  return a2 / (a2 + b2);
}

// ---------------------------------------------------------------------------
// Golf-ball displaced sphere surface (shaders/shader_golf.cu:53-140): the hit
// distance is the base sphere's; position and normal are displaced here.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float golf_dimple(const f3 &p) {
  const f3 q = normalize(p);
  const int N = 150;
  float best = -1.0f;
  for (int i = 0; i < N; ++i) best = fmaxf(best, dot(q, fib_point(i, N)));
  best = fmaxf(fminf(best, 1.0f), -1.0f);
  const float ang = acosf(best);
  const float radius = 0.24f, depth = 0.35f;
  if (ang < radius) return -depth * cosf((ang / radius) * RB_PI * 0.5f);
  return 0.0f;
}

static __device__ __noinline__ Surface golf_surface(const f3 &center, float radius, const Ray &r, float t) {
  Surface s;
  s.center = center;
  const f3 sp = r.at(t);
  {
    const f3 outward = (sp - center) / radius;
    f3 tg = cross(f3(0.0f, 1.0f, 0.0f), outward);
    if (tg.length_squared() < 1e-6f) tg = f3(1.0f, 0.0f, 0.0f);
    s.tangent = normalize(tg);
  }
  const float disp = golf_dimple(normalize(sp - center));
  const f3 base_out = normalize(sp - center);
  const float dn = fminf(1.0f, fmaxf(0.0f, -disp / 0.35f));
  const float push = radius * 0.35f * (1.0f - dn);
  f3 p = sp + base_out * push;
  const f3 bn = normalize(p - center);
  f3 n = bn;
  if (disp < -0.001f) {
    const f3 helper = fabsf(bn.x) > 0.8f ? f3(0, 1, 0) : f3(1, 0, 0);
    const f3 t1 = normalize(cross(helper, bn));
    const f3 t2 = cross(bn, t1);
    const float h = 0.015f;
    const float g0 = golf_dimple(bn);
    const float g1 = golf_dimple(normalize(bn + h * t1));
    const float g2 = golf_dimple(normalize(bn + h * t2));
    const float dd1 = (g1 - g0) / h, dd2 = (g2 - g0) / h;
    f3 dnv = -0.2f * (dd1 * t1 + dd2 * t2);
    const f3 view = normalize(-r.d);
    const float ndv = fmaxf(0.0f, dot(bn, view));
    const float x = fmaxf(0.0f, fminf(1.0f, (ndv - 0.1f) / 0.3f));
    dnv = dnv * (x * x * (3.0f - 2.0f * x));
    const float len = dnv.length();
    if (len > 0.4f && len > 1e-6f) dnv = (0.4f / len) * dnv;
    f3 pert = normalize(bn + dnv);
    if (dot(pert, bn) < 0.0f) pert = -pert;
    if (!(pert.x == pert.x) || !(pert.y == pert.y) || !(pert.z == pert.z)) pert = bn;
    n = pert;
  }
  float ndv = dot(r.d, n);
  if (!(ndv == ndv)) {
    n = bn;
    ndv = dot(r.d, n);
  }
  s.front = ndv < 0;
  if (!s.front) n = -n;
  s.n = n;
  s.p = p + n * 1e-3f;
  return s;
}

// ---------------------------------------------------------------------------
// SDF primitives (sphere tracing; distance functions after
// cpu_renderers/cpu_shapes/sdf.hpp:105-160, 410-416, 499-566)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sdf_eval1(const SdfPrim &q, const f3 &pw) {
  const f3 d0 = pw - f3(q.px, q.py, q.pz);
  const f3 p(q.r00 * d0.x + q.r01 * d0.y + q.r02 * d0.z, q.r10 * d0.x + q.r11 * d0.y + q.r12 * d0.z,
             q.r20 * d0.x + q.r21 * d0.y + q.r22 * d0.z);
  switch (q.type) {
    case 0:  // sphere
      return p.length() - q.a;
    case 1:    // box
    case 32: {  // rounded box
      const f3 qq(fabsf(p.x) - (q.a - q.round), fabsf(p.y) - (q.b - q.round), fabsf(p.z) - (q.c - q.round));
      const float outside = f3(fmaxf(qq.x, 0.0f), fmaxf(qq.y, 0.0f), fmaxf(qq.z, 0.0f)).length();
      const float inside = fminf(fmaxf(qq.x, fmaxf(qq.y, qq.z)), 0.0f);
      return outside + inside - q.round;
    }
    case 2: {  // torus (major a, minor b) in the local XZ plane
      const float qx = sqrtf(p.x * p.x + p.z * p.z) - q.a;
      return sqrtf(qx * qx + p.y * p.y) - q.b;
    }
    case 3: {  // capsule: radius a, height b along local y, centred
      const float hh = q.b * 0.5f;
      const float y = fminf(fmaxf(p.y, -hh), hh);
      return f3(p.x, p.y - y, p.z).length() - q.a;
    }
    default:
      return 1e30f;
  }
}

// sdf_eval1 of a record given as its five 16-byte words.
__device__ __forceinline__ float sdf_eval_words(const float4 &w0, const float4 &w1, const float4 &w2, const float4 &w3,
                                                const float4 &w4, const f3 &pw) {
  SdfPrim q;
  q.px = w0.x; q.py = w0.y; q.pz = w0.z; q.a = w0.w;
  q.b = w1.x; q.c = w1.y; q.round = w1.z; q.type = __float_as_int(w1.w);
  q.r00 = w2.x; q.r01 = w2.y; q.r02 = w2.z; q.r10 = w2.w;
  q.r11 = w3.x; q.r12 = w3.y; q.r20 = w3.z; q.r21 = w3.w;
  q.r22 = w4.x;
  return sdf_eval1(q, pw);
}

// sdf_eval1 of primitive i of the table, its record read as five 128-bit loads.
__device__ __forceinline__ float sdf_eval_at(const SdfPrim *__restrict__ tab, int i, const f3 &pw) {
  const float4 *v = reinterpret_cast<const float4 *>(tab + i);
  return sdf_eval_words(__ldg(v), __ldg(v + 1), __ldg(v + 2), __ldg(v + 3), __ldg(v + 4), pw);
}

__device__ __forceinline__ float smin_poly(float d1, float d2, float k) {
  const float h = fminf(fmaxf(0.5f + 0.5f * (d2 - d1) / k, 0.0f), 1.0f);
  return d2 * (1.0f - h) + d1 * h - k * h * (1.0f - h);
}

// Smooth-union field of the collected SDF primitives: polynomial smooth
// minimum (sdf.hpp:410-416) folded in primitive-index order. A primitive takes
// part where the ray is inside its k-inflated bounding sphere (its window
// [t0, t1]); outside, its distance is at least k, so folding it would not
// move the union's surface. Sphere tracing on the field's magnitude (a ray
// that starts inside marches to the exit), each step clamped to the next
// window entry so no primitive is stepped over, at most S.sdf_steps steps,
// hit below S.sdf_eps; outward normal by central differences with a 5e-4 step
// over the hit point's window set; the material is that of the nearest
// primitive.
//
// Convex skip: where one window alone holds t and its primitive is convex
// (sphere, box, rounded box, capsule), the field is that primitive's distance,
// a convex function of t. Once it has grown between two consecutive steps by
// more than a quarter (a margin FP32 rounding near the surface cannot fake),
// it keeps growing, so no hit lies before the next window entry and the march
// jumps there (where it would have arrived, clamped, after more steps). Rays
// leaving a surface and rays past their closest approach stop crawling.
#define RB_SDF_NORMAL_EPS 5e-4f
#define RB_SDF_FAR 1e30f
#ifndef RB_SDF_SKIP_GROWTH
#define RB_SDF_SKIP_GROWTH 1.25f
#endif
// Field at p = r.at(t) over the windows holding t; `next` is the nearest
// window entry beyond t (RB_SDF_FAR when none). RB_SDF_FAR when no window
// holds t. `lone` (optional) gets the candidate code of the only window
// holding t, -1 when none or several do.
__device__ __forceinline__ float sdf_field_eval(const SceneView &S, const SdfCand &c, const f3 &p, float t,
                                                float &next, int *nearest, int *lone = nullptr) {
  // two passes so that a warp's lanes evaluate together: mark the candidates
  // whose window holds t (index order), then fold the marked ones
  uint32_t active = 0;
  next = RB_SDF_FAR;
  for (int i = 0; i < c.n; ++i) {
    const float t0 = c.t0[i];
    if (t0 > t) next = fminf(next, t0);
    else if (t <= c.t1[i]) active |= 1u << i;
  }
  if (lone) *lone = (active != 0u && (active & (active - 1u)) == 0u) ? c.idx[__ffs(active) - 1] : -1;
  float F = RB_SDF_FAR, best = RB_SDF_FAR;
  bool first = true;
  while (active) {
    const int i = __ffs(active) - 1;
    active &= active - 1;
    const int id = c.idx[i] >> 1;
    const float d = sdf_eval_at(S.sdf, id, p);
    if (nearest && d < best) {
      best = d;
      *nearest = id;
    }
    F = first ? d : smin_poly(F, d, S.sdf_k);
    first = false;
  }
  return F;
}

// Candidates sorted by primitive index (insertion sort) so the fold order is fixed.
__device__ __forceinline__ void sdf_sort_cand(SdfCand &c) {
  for (int i = 1; i < c.n; ++i) {
    const int v = c.idx[i];
    const float a0 = c.t0[i], a1 = c.t1[i];
    int j = i - 1;
    while (j >= 0 && c.idx[j] > v) {
      c.idx[j + 1] = c.idx[j];
      c.t0[j + 1] = c.t0[j];
      c.t1[j + 1] = c.t1[j];
      --j;
    }
    c.idx[j + 1] = v;
    c.t0[j + 1] = a0;
    c.t1[j + 1] = a1;
  }
}

static __device__ __noinline__ bool sdf_field_march(const SceneView &S, const Ray &r, float tmin, float tmax,
                                                    SdfCand &c, float &t_out, f3 &n_out, int &mat_out) {
  sdf_sort_cand(c);
  const float inv_len = 1.0f / r.d.length();
  float t = tmin, next;
  int lone = -1;
  // a ray that starts in the eps shell around the surface (a bounce off the
  // field) first steps out of it, so the inside/outside decision is made
  // where the field is clearly signed
  float raw = sdf_field_eval(S, c, r.at(t), t, next, nullptr, &lone);
  for (int k = 0; k < 8 && fabsf(raw) < 2.0f * S.sdf_eps; ++k) {
    t += 2.0f * S.sdf_eps * inv_len;
    raw = sdf_field_eval(S, c, r.at(t), t, next, nullptr, &lone);
  }
  const float sgn = raw < 0.0f ? -1.0f : 1.0f;
  int prev = -1;  // lone convex candidate of the previous step, and the field there
  float prev_d = 0.0f;
  for (int i = 0; i < S.sdf_steps; ++i) {
    const f3 p = r.at(t);
    // the last escape evaluation is the first step's
    if (i > 0) raw = sdf_field_eval(S, c, p, t, next, nullptr, &lone);
    if (raw == RB_SDF_FAR) {  // between windows: jump to the next entry
      if (next == RB_SDF_FAR || next > tmax) return false;
      t = next;
      prev = -1;
      continue;
    }
    const float F = sgn * raw;
    if (F < S.sdf_eps) {
      if (t > tmax) return false;
      const float e = RB_SDF_NORMAL_EPS;
      float nx;
      const f3 g(sdf_field_eval(S, c, p + f3(e, 0, 0), t, nx, nullptr) -
                     sdf_field_eval(S, c, p - f3(e, 0, 0), t, nx, nullptr),
                 sdf_field_eval(S, c, p + f3(0, e, 0), t, nx, nullptr) -
                     sdf_field_eval(S, c, p - f3(0, e, 0), t, nx, nullptr),
                 sdf_field_eval(S, c, p + f3(0, 0, e), t, nx, nullptr) -
                     sdf_field_eval(S, c, p - f3(0, 0, e), t, nx, nullptr));
      const float gl = g.length();
      n_out = gl > 0.0f ? g / gl : f3(0.0f, 1.0f, 0.0f);
      int nearest = c.idx[0] >> 1;
      sdf_field_eval(S, c, p, t, nx, &nearest);
      mat_out = S.sdf[nearest].material;
      t_out = t;
      return true;
    }
    const int one = (sgn > 0.0f && lone >= 0 && (lone & 1)) ? lone : -1;
    if (one >= 0 && one == prev && raw > RB_SDF_SKIP_GROWTH * prev_d) {  // convex skip
      if (next == RB_SDF_FAR || next > tmax) return false;
      t = next;
      prev = -1;
      continue;
    }
    prev = one;
    prev_d = raw;
    t = fminf(t + F * inv_len, next);
    if (t > tmax) return false;
  }
  return false;
}

// Single hard-union SDF primitive marched on its own (closest-hit test through
// the BVH); returns t or -1.
static __device__ __noinline__ float sdf_march_prim(const SceneView &S, int prim, const Ray &r, float tmin, float tmax) {
  const float4 *pr = S.prims + 3 * (size_t)prim;
  const float4 a = __ldg(pr), b = __ldg(pr + 1);
  const SdfPrim q = S.sdf[__float_as_int(b.x)];
  // start at the bounding sphere entry
  float t0;
  if (!t_sphere(f3(a.x, a.y, a.z), a.w, r, tmin, tmax, t0)) {
    // origin inside the bound: march from tmin
    const f3 oc = r.o - f3(a.x, a.y, a.z);
    if (dot(oc, oc) > a.w * a.w) return -1.0f;
    t0 = tmin;
  }
  const float inv_len = 1.0f / r.d.length();
  float t = t0;
  for (int i = 0; i < S.sdf_steps; ++i) {
    const float dist = sdf_eval1(q, r.at(t));
    if (dist < S.sdf_eps) return (t >= tmin && t <= tmax) ? t : -1.0f;
    t += dist * inv_len;
    if (t > tmax) return -1.0f;
  }
  return -1.0f;
}

static __device__ __noinline__ Surface sdf_surface(const SceneView &S, int prim, const Ray &r, float t) {
  const float4 *pr = S.prims + 3 * (size_t)prim;
  const float4 b = __ldg(pr + 1);
  const SdfPrim q = S.sdf[__float_as_int(b.x)];
  Surface s;
  s.p = r.at(t);
  const float e = S.sdf_eps;
  const f3 g(sdf_eval1(q, s.p + f3(e, 0, 0)) - sdf_eval1(q, s.p - f3(e, 0, 0)),
             sdf_eval1(q, s.p + f3(0, e, 0)) - sdf_eval1(q, s.p - f3(0, e, 0)),
             sdf_eval1(q, s.p + f3(0, 0, e)) - sdf_eval1(q, s.p - f3(0, 0, e)));
  f3 n = normalize(g);
  s.front = dot(r.d, n) < 0;
  s.n = s.front ? n : -n;
  f3 tg = cross(f3(0.0f, 1.0f, 0.0f), n);
  if (tg.length_squared() < 1e-6f) tg = f3(1.0f, 0.0f, 0.0f);
  s.tangent = normalize(tg);
  s.center = f3(q.px, q.py, q.pz);
  return s;
}

}  // namespace rbd
