// Path construction shared by the per-frame kernel and the batched engine:
// camera rays, one path segment (trace, shade, next-event estimation, Russian
// roulette) and compensated accumulation.
#pragma once

#include "rb_internal.hpp"

namespace rb {

using namespace rbd;

__device__ __forceinline__ void kahan_add(float &sum, float &c, float x) {
  const float y = __fsub_rn(x, c);
  const float t = __fadd_rn(sum, y);
  c = __fsub_rn(__fsub_rn(t, sum), y);
  sum = t;
}

// Camera ray of one sample (render_acc_kernel.cu:198-222); lens by polar mapping.
__device__ __forceinline__ Ray camera_ray(const FrameF &P, const Globals &G, int x, int y, uint32_t key) {
  const float ou = rb_draw(key, RB_DIM_JITTER) - 0.5f;
  const float ov = rb_draw(key, RB_DIM_JITTER + 1) - 0.5f;
  const f3 pc = P.p00 + ((float)x + ou) * P.du + ((float)y + ov) * P.dv;
  Ray r;
  r.o = P.center;
  r.d = pc - P.center;
  if (G.dof_enabled && G.dof_aperture > 0.0f) {
    const f3 nd = normalize(r.d);
    const f3 focus = P.center + G.dof_focus * nd;
    const float rr = sqrtf(rb_draw(key, RB_DIM_LENS));
    float s, c;
    __sincosf(2.0f * RB_PI * rb_draw(key, RB_DIM_LENS + 1), &s, &c);
    const f3 off = G.dof_aperture * ((rr * c) * P.cu + (rr * s) * P.cv);
    r.o = P.center + off;
    r.d = focus - r.o;
  }
  return r;
}

// One path segment: trace, shade, NEE, Russian roulette. Returns true when the
// path ended (radiance complete in L).
template <bool NEE, int MS, int NODES = RB_NODES_ANY>
__device__ __forceinline__ bool path_segment(const SceneView &S, const Globals &G, Stack &st, uint32_t &ovf, Ray &ray,
                                             f3 &thr, f3 &L, int &bounce, float &prev_pdf, uint32_t key,
                                             int max_depth) {
  const HitInfo h = trace<false, MS, RB_SPEC_TRAVERSAL, NODES>(S, ray, 0.001f, FLT_MAX, st, ovf);
  if (h.prim == -1) {  // miss (-2 is a hit on the smooth SDF field)
    if (G.background_intensity != 0.0f) L = L + thr * sky(ray.d) * G.background_intensity;
    return true;
  }
  const Surface sf = surface<MS>(S, ray, h);
  if (!sf.visible && bounce == 0) {  // camera rays pass through invisible geometry
    ray.o = sf.p + ray.d * 0.01f;
    return ++bounce >= max_depth;
  }
  if (sf.mat >= S.num_mats) return true;
  const DevMaterial &m = S.mats[sf.mat];
  const ScatterOut so = scatter<MS>(G, m, sf, ray, key, bounce);
  if (so.emit.length_squared() > 0.0f) {
    float w = 1.0f;
    if (NEE && G.nee && prev_pdf > 0.0f && m.kind == L_LIGHT && S.num_lights > 0) {
      // MIS weight of the BSDF strategy for an emitter that NEE also samples
      const float dl = h.t * ray.d.length();
      const f3 ud = normalize(ray.d);
      f3 gn = sf.n;  // |cos| at the light only needs the line, not the side
      const float cl = fabsf(dot(gn, ud));
      const float pl = cl > 0.0f ? dl * dl / (cl * S.light_area) : 0.0f;
      w = mis2(prev_pdf, pl);
    }
    L = L + thr * so.emit * w;
  }
  if (!so.scattered) return true;
  if (NEE && G.nee) {
    prev_pdf = 0.0f;
    if (m.kind == L_LAMBERTIAN && bounce + 1 < max_depth && S.num_lights > 0) {
      LightSample ls;
      const uint32_t dl = rb_vdim(bounce, RB_SLOT_LIGHT);
      if (sample_light(S, G, rb_draw(key, dl), rb_draw(key, dl + 1), rb_draw(key, dl + 2), ls)) {
        const f3 o = so.ray.o;
        const f3 dv = ls.p - o;
        const float d2 = dv.length_squared();
        const float dist = sqrtf(d2);
        const f3 wi = dv / dist;
        const f3 nn = normalize(sf.n);
        const float cs = dot(nn, wi);
        const float cl = fabsf(dot(ls.n, wi));
        if (cs > 0.0f && cl > 0.0f) {
          Ray sr;
          sr.o = o;
          sr.d = wi;
          const HitInfo sh = trace<true, MS, RB_SPEC_TRAVERSAL, NODES>(S, sr, 0.001f, dist * (1.0f - 1e-4f), st, ovf);
          if (sh.prim == -1) {  // unoccluded
            const float pl = d2 / (cl * S.light_area);
            const float pb = cs * (1.0f / RB_PI);
            const float w = mis2(pl, pb);
            // f * Le * cos / pdf_l with f = albedo / pi; the albedo is the scatter attenuation
            L = L + thr * so.att * ls.Le * (cs * (1.0f / RB_PI) * w / pl);
          }
        }
      }
      prev_pdf = so.pdf;
    }
  }
  thr = thr * so.att;
  if (bounce > 0) {
    const float mc = fmaxf(thr.x, fmaxf(thr.y, thr.z));
    const float sp = fminf(mc, 0.95f);
    if (rb_draw(key, rb_vdim(bounce, RB_SLOT_RR)) > sp) return true;
    thr = thr / sp;
  }
  ray = so.ray;
  return ++bounce >= max_depth;
}


}  // namespace rb
