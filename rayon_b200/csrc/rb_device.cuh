// Device side of the B200 render path: layout, intersection, traversal,
// surface reconstruction and material scatter.
//
// Arithmetic that decides WHICH primitive a ray hits (box slabs, sphere,
// quad and triangle tests, the closest-hit update rule and the traversal
// order) is written operation for operation as in
// src/rayon/gpu_renderers/cuda_raytracer.cuh:154-347, 487-602 and compiled
// with the same fast-math flags, so primary-hit ids are bit-exact against
// the reference. Everything after the hit (shading, sampling) is this
// project's own and is checked statistically against the FP64 oracle.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "rb_rng.h"

namespace rbd {

// ---------------------------------------------------------------------------
// float3 algebra (expression shapes follow cuda_float3.cuh:41-96)
// ---------------------------------------------------------------------------
struct f3 {
  float x, y, z;
  __host__ __device__ __forceinline__ f3() {}
  __host__ __device__ __forceinline__ f3(float a, float b, float c) : x(a), y(b), z(c) {}
  __host__ __device__ __forceinline__ f3 operator+(const f3 &o) const { return f3(x + o.x, y + o.y, z + o.z); }
  __host__ __device__ __forceinline__ f3 operator-(const f3 &o) const { return f3(x - o.x, y - o.y, z - o.z); }
  __host__ __device__ __forceinline__ f3 operator*(float t) const { return f3(x * t, y * t, z * t); }
  __host__ __device__ __forceinline__ f3 operator*(const f3 &o) const { return f3(x * o.x, y * o.y, z * o.z); }
  __host__ __device__ __forceinline__ f3 operator/(float t) const { return f3(x / t, y / t, z / t); }
  __host__ __device__ __forceinline__ f3 operator-() const { return f3(-x, -y, -z); }
  __host__ __device__ __forceinline__ float length() const { return sqrtf(x * x + y * y + z * z); }
  __host__ __device__ __forceinline__ float length_squared() const { return x * x + y * y + z * z; }
};
__device__ __forceinline__ f3 operator*(float t, const f3 &v) { return v * t; }
__device__ __forceinline__ float dot(const f3 &a, const f3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(const f3 &a, const f3 &b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ f3 normalize(const f3 &v) { return v / v.length(); }
__device__ __forceinline__ f3 mk(float4 v) { return f3(v.x, v.y, v.z); }

struct Ray {
  f3 o, d;
  __device__ __forceinline__ f3 at(float t) const { return o + t * d; }
};

// ---------------------------------------------------------------------------
// Device layout
// ---------------------------------------------------------------------------
// Primitive record: 3 x float4 = 48 B. Word 11 is the tag:
//   bits 0-2 kind, bit 3 visible, bit 4 has vertex normals, bits 8-31 material.
//   SPHERE / DISPLACED: f0 = (centre, radius)
//   RECT:               f0 = (corner, u.x) f1 = (u.y, u.z, v.x, v.y) f2.x = v.z
//   TRI:                f0 = (v0, e1.x)    f1 = (e1.y, e1.z, e2.x, e2.y) f2.x = e2.z
//   SDF:                f0 = (bounding centre, bounding radius), f1.x = index into sdf table
enum PrimKind : uint32_t { PK_SPHERE = 0, PK_RECT = 1, PK_TRI = 2, PK_DISPLACED = 3, PK_SDF = 4, PK_NONE = 7 };
__device__ __host__ __forceinline__ uint32_t tag_kind(uint32_t t) { return t & 7u; }
__device__ __host__ __forceinline__ bool tag_visible(uint32_t t) { return (t >> 3) & 1u; }
__device__ __host__ __forceinline__ bool tag_normals(uint32_t t) { return (t >> 4) & 1u; }
__device__ __host__ __forceinline__ int tag_material(uint32_t t) { return (int)(t >> 8); }

// BVH2 node with both child boxes (64 B):
//   f0 = (L.min.xyz, L.max.x) f1 = (L.max.yz, R.min.xy) f2 = (R.min.z, R.max.xyz)
//   f3 = (left ref, right ref, split axis, 0) as int bits.
// A child ref >= 0 is an interior node; a leaf ref has bit 31 set,
// (count - 1) in bits 26-30 and the first primitive in bits 0-25.
__device__ __host__ __forceinline__ bool ref_is_leaf(int r) { return r < 0; }
__device__ __host__ __forceinline__ int leaf_first(int r) { return r & 0x03FFFFFF; }
__device__ __host__ __forceinline__ int leaf_count(int r) { return ((r >> 26) & 31) + 1; }
__host__ __forceinline__ int make_leaf_ref(int first, int count) {
  return (int)(0x80000000u | ((uint32_t)(count - 1) << 26) | (uint32_t)first);
}

// Quantised node: 32 B, one 32-byte sector per visit (the FP32 two-box node
// is 64 B, two sectors). A grid anchored at the union box's minimum corner,
// with a power-of-two step per axis, holds 8-bit child bounds rounded outward
// (min down, max up), so the decoded box always contains the FP32 child box.
//   ox, oy, oz: bits 31-8 = the corner coordinate's FP32 bits with the low 8
//               mantissa bits dropped, rounded toward -inf; bits 7-1 = the
//               axis's step exponent + 64; bit 0 of ox, oy = the split axis
//   lq0 = L lo xyz, L hi x;  lq1 = L hi yz, R lo xy;  rq = R lo z, R hi xyz
//   left, right: child refs
struct __align__(16) QNode {
  uint32_t ox, oy, oz;
  uint32_t lq0, lq1, rq;
  int left;
  int right;
};
static_assert(sizeof(QNode) == 32, "a quantised node is one 32-byte sector");

// The grid corner and step of one axis word of a quantised node.
__device__ __host__ __forceinline__ float qnode_origin(uint32_t w) {
  const uint32_t b = w & 0xFFFFFF00u;
  float f;
  memcpy(&f, &b, 4);
  return f;
}
__device__ __host__ __forceinline__ float qnode_step(uint32_t w) {
  const uint32_t b = (((w >> 1) & 0x7Fu) + 63u) << 23;  // 2^(stored - 64)
  float f;
  memcpy(&f, &b, 4);
  return f;
}

// Legacy material kinds of the reference shader (cuda_raytracer.cuh:43-55).
enum Legacy : int {
  L_LAMBERTIAN = 0, L_MIRROR = 1, L_GLASS = 2, L_LIGHT = 3, L_ROUGH_MIRROR = 4, L_CONSTANT = 5,
  L_SHOW_NORMALS = 6, L_ANISO_METAL = 7, L_THIN_FILM = 8, L_CLEAR_COAT = 9, L_ABSORB = 15
};

// Material after the reference's apply_material mapping (cuda_raytracer.cuh:418-485):
// kind, colour, roughness defaults and IOR rules resolved on the host.
struct __align__(16) DevMaterial {
  int kind;
  int pattern;         // 0 none, 1 Fibonacci dots
  float roughness;
  float ior;           // per-material IOR (clear coat, thin film exterior)
  f3 color;
  float anisotropy;
  f3 emission;
  float film_thickness;
  f3 eta;
  float film_ior;
  f3 k;
  float pattern_p1;
  f3 pattern_color;
  float pattern_p2;
};

struct LightRec {      // one emitter sampled by next-event estimation
  int prim;
  float area;
  float cdf;           // inclusive CDF over area
  float pad;
};

// One SDF primitive (ray marched): 5 x 16 B, read by the field march as five
// 128-bit loads. Position, parameters a b c, rounding radius (ROUND_BOX),
// type, world->local rotation r00..r22, material.
// Kernel parameters that device functions take by reference stay in the
// parameter space (no per-thread copy into local memory). Used where it was
// measured to pay: the wavefront extend kernel (one ray per thread: 2.20 ->
// 2.03 ms per launch on the SDF field, local stores halved) and the
// per-frame and primary-hit kernels; the shade kernel ran 14 % slower with it.
#ifndef RB_GRID_CONST
#define RB_GRID_CONST __grid_constant__
#endif

struct __align__(16) SdfPrim {
  float px, py, pz, a;
  float b, c, round;
  int type;
  float r00, r01, r02, r10;
  float r11, r12, r20, r21;
  float r22;
  int material;
  float bound_r;  // the k-inflated bounding-sphere radius (centre px, py, pz)
  int convex;     // 1: distance convex along a ray (sphere, box, rounded box, capsule)
};
static_assert(sizeof(SdfPrim) == 80, "SdfPrim is five 16-byte words");

// Kernel-parameter view of a device scene (passed by value).
struct SceneView {
  const float4 *__restrict__ nodes;
  const QNode *__restrict__ qnodes;
  const float4 *__restrict__ wnodes;  // 4-wide copy of the tree (render kernels) or null
  const float4 *__restrict__ prims;
  const float4 *__restrict__ normals;  // 3 x float4 per primitive or null
  const DevMaterial *__restrict__ mats;
  const LightRec *__restrict__ lights;
  const SdfPrim *__restrict__ sdf;
  const float4 *__restrict__ groups;  // 2 per group: (box min, first primitive), (box max, count)
  int num_groups;                     // > 0: grouped linear layout (no BVH traversal)
  int root_ref;
  int num_prims;
  int num_mats;
  int num_lights;
  int use_bvh;
  int quantized;
  int num_sdf;
  int sdf_steps;
  float root_box[6];
  float light_area;    // total emitter area
  float sdf_k;         // smooth-union radius
  float sdf_eps;
  int trav_budget;     // traversal step budget override (0: 2 * (prims + 4) + 64)
  int short_stack;     // traversal stack entries in shared memory (0: RB_SHORT)
  int wide_root;       // root of wnodes
  // Rays whose traversal ran out of its step budget (a corrupt tree; never a
  // well-formed one): counted here, read by rb_scene_traversal_faults.
  unsigned long long *faults;
};

__device__ __forceinline__ int traversal_budget(const SceneView &S) {
  return S.trav_budget > 0 ? S.trav_budget : 2 * (S.num_prims + 4) + 64;
}

__device__ __forceinline__ void note_budget_exhausted(const SceneView &S, int budget) {
  if (budget <= 0 && S.faults) atomicAdd(S.faults, 1ull);
}

// Reference __constant__ settings (renderer_cuda_device.cu:18-26), passed by value.
struct Globals {
  float light_intensity;
  float background_intensity;
  float metal_fuzziness;
  float glass_ior;
  int dof_enabled;
  float dof_aperture;
  float dof_focus;
  int nee;
};

// ---------------------------------------------------------------------------
// Ray / box (hit_aabb, cuda_raytracer.cuh:154-197)
// ---------------------------------------------------------------------------
struct RayPre {
  f3 o, d, inv;
};
__device__ __forceinline__ RayPre prep(const Ray &r) {
  RayPre p;
  p.o = r.o;
  p.d = r.d;
  p.inv = f3(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
  return p;
}

// Slab test. Swapping t0/t1 when inv < 0 is the same as taking the max bound as
// the near plane, so the values compared are those of the reference.
__device__ __forceinline__ bool box_hit(const RayPre &r, float x0, float y0, float z0, float x1, float y1,
                                        float z1, float tmin, float tmax, float &tenter) {
  float t0x = (x0 - r.o.x) * r.inv.x, t1x = (x1 - r.o.x) * r.inv.x;
  if (r.inv.x < 0.0f) { float t = t0x; t0x = t1x; t1x = t; }
  float t0y = (y0 - r.o.y) * r.inv.y, t1y = (y1 - r.o.y) * r.inv.y;
  if (r.inv.y < 0.0f) { float t = t0y; t0y = t1y; t1y = t; }
  float t0z = (z0 - r.o.z) * r.inv.z, t1z = (z1 - r.o.z) * r.inv.z;
  if (r.inv.z < 0.0f) { float t = t0z; t0z = t1z; t1z = t; }
  const float te = fmaxf(fmaxf(t0x, t0y), t0z);
  const float tx = fminf(fminf(t1x, t1y), t1z);
  tenter = te;
  return te <= tx && tx >= tmin && te <= tmax;
}

// ---------------------------------------------------------------------------
// Primitive tests returning only t (cuda_raytracer.cuh:203-347)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool t_sphere(const f3 &center, float radius, const Ray &r, float tmin, float tmax,
                                         float &tout) {
  f3 oc = r.o - center;
  float a = dot(r.d, r.d);
  float half_b = dot(oc, r.d);
  float c = dot(oc, oc) - radius * radius;
  float disc = half_b * half_b - a * c;
  if (disc < 0) return false;
  float sqrtd = sqrtf(disc);
  float root = (-half_b - sqrtd) / a;
  if (root < tmin || tmax < root) {
    root = (-half_b + sqrtd) / a;
    if (root < tmin || tmax < root) return false;
  }
  tout = root;
  return true;
}

__device__ __forceinline__ bool t_rect(const f3 &corner, const f3 &u, const f3 &v, const Ray &r, float tmin,
                                       float tmax, float &tout) {
  f3 normal = normalize(f3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x));
  float denom = dot(normal, r.d);
  if (fabsf(denom) < 1e-8f) return false;
  float t = dot(normal, corner - r.o) / denom;
  if (t < tmin || t > tmax) return false;
  f3 p = r.at(t) - corner;
  float alpha = dot(p, u) / dot(u, u);
  float beta = dot(p, v) / dot(v, v);
  if (alpha < 0.0f || alpha > 1.0f || beta < 0.0f || beta > 1.0f) return false;
  tout = t;
  return true;
}

// Moller-Trumbore with the reference's comparisons; edges are stored
// precomputed (e1 = v1 - v0, e2 = v2 - v0 in FP32, the values the reference
// computes per test).
__device__ __forceinline__ bool t_tri(const f3 &v0, const f3 &edge1, const f3 &edge2, const Ray &r, float tmin,
                                      float tmax, float &tout) {
  const f3 h = cross(r.d, edge2);
  const float a = dot(edge1, h);
  if (fabsf(a) < 1e-8f) return false;
  const float f = 1.0f / a;
  const f3 s = r.o - v0;
  const float u = f * dot(s, h);
  if (u < 0.0f || u > 1.0f) return false;
  const f3 q = cross(s, edge1);
  const float v = f * dot(r.d, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  const float t = f * dot(edge2, q);
  if (t < tmin || t > tmax) return false;
  tout = t;
  return true;
}

static __device__ float sdf_march_prim(const SceneView &S, int prim, const Ray &r, float tmin, float tmax);

// SDF primitives of a smooth-union scene (blend radius k > 0) are not hit one
// by one: a ray collects the ones whose k-inflated bounding spheres it crosses,
// each with the ray interval [t0, t1] inside its sphere, and the union field
// of those is sphere-traced after the traversal.
#define RB_SDF_CAND 24
static_assert(RB_SDF_CAND <= 32, "field folds mark candidates in a 32-bit mask");
// idx[i] is a candidate code: (SDF table index << 1) | 1 when the primitive is
// convex. Codes order as their indices do.
struct SdfCand {
  int n;
  int idx[RB_SDF_CAND];
  float t0[RB_SDF_CAND], t1[RB_SDF_CAND];
  // code = SDF table index << 1 | convex flag; window [t0, t1] along the ray
  __device__ __forceinline__ void add(int code, float a0, float a1) {
    if (n < RB_SDF_CAND) {
      idx[n] = code;
      t0[n] = a0;
      t1[n] = a1;
      ++n;
    }
  }
};

// The wavefront engine's candidate set: one bit per SDF table entry (tables of
// at most RB_SDF_MASK_BITS primitives), kept in registers. Index order comes
// for free (no per-ray arrays, no sort) and the set has no size cap; the
// march recomputes each window from the primitive's bounding sphere.
#define RB_SDF_MASK_WORDS 8
#define RB_SDF_MASK_BITS (32 * RB_SDF_MASK_WORDS)
struct SdfMask {
  uint32_t w[RB_SDF_MASK_WORDS];
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int k = 0; k < RB_SDF_MASK_WORDS; ++k) w[k] = 0u;
  }
  __device__ __forceinline__ void add(int code, float, float) {
    const int i = code >> 1;
    const uint32_t bit = 1u << (i & 31);
#pragma unroll
    for (int k = 0; k < RB_SDF_MASK_WORDS; ++k)
      if (k == (i >> 5)) w[k] |= bit;  // static indices: the words stay in registers
  }
  __device__ __forceinline__ bool any() const {
    uint32_t a = 0u;
#pragma unroll
    for (int k = 0; k < RB_SDF_MASK_WORDS; ++k) a |= w[k];
    return a != 0u;
  }
};

// The closest-hit test of primitive i given its record's three words.
template <int MS, class Sink = SdfCand>
__device__ __forceinline__ bool prim_t_words(const SceneView &S, int i, const float4 &a, const float4 &b,
                                             const float4 &c, const Ray &r, float tmin, float tmax, float &t,
                                             Sink *cand = nullptr) {
  const uint32_t tag = __float_as_uint(c.w);
  const uint32_t kind = tag_kind(tag);
  if (kind == PK_SPHERE || kind == PK_DISPLACED) return t_sphere(f3(a.x, a.y, a.z), a.w, r, tmin, tmax, t);
  if (kind == PK_TRI)
    return t_tri(f3(a.x, a.y, a.z), f3(a.w, b.x, b.y), f3(b.z, b.w, c.x), r, tmin, tmax, t);
  if (kind == PK_RECT)
    return t_rect(f3(a.x, a.y, a.z), f3(a.w, b.x, b.y), f3(b.z, b.w, c.x), r, tmin, tmax, t);
  if (MS >= 4 && kind == PK_SDF) {
    if (cand) {
      // collect when the inflated bounding sphere overlaps [tmin, tmax]
      const f3 oc = r.o - f3(a.x, a.y, a.z);
      const float aa = dot(r.d, r.d), hb = dot(oc, r.d), cc = dot(oc, oc) - a.w * a.w;
      const float disc = hb * hb - aa * cc;
      if (disc >= 0.0f) {
        const float sq = sqrtf(disc);
        const float t0 = (-hb - sq) / aa, t1 = (-hb + sq) / aa;
        if (t1 >= tmin && t0 <= tmax) cand->add((__float_as_int(b.x) << 1) | (__float_as_int(b.y) & 1), t0, t1);
      }
      return false;
    }
    const float ts = sdf_march_prim(S, i, r, tmin, tmax);
    if (ts >= 0.0f) { t = ts; return true; }
  }
  return false;
}

// The test with the record loaded here: all three words in one round trip
// (the kind tag is in the last word; loading the middle word only after
// testing it would put a second dependent memory latency on every triangle
// and quad test).
template <int MS, class Sink = SdfCand>
__device__ __forceinline__ bool prim_t(const SceneView &S, int i, const Ray &r, float tmin, float tmax,
                                       float &t, Sink *cand = nullptr) {
  const float4 *p = S.prims + 3 * (size_t)i;
  const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  return prim_t_words<MS, Sink>(S, i, a, b, c, r, tmin, tmax, t, cand);
}


// ---------------------------------------------------------------------------
// Traversal (hit_scene, cuda_raytracer.cuh:487-602)
// ---------------------------------------------------------------------------
// The reference pops a node, tests its box against the current closest t and
// pushes (far, near) by the sign of the ray on the node's split axis. Here the
// parent holds both child boxes: each child is tested when its parent is
// visited. The near child would be popped next in the reference with the same
// closest t, so its result is identical. The far child is pushed with its
// entry distance and re-checked against the closest t when popped; the other
// two conditions of the slab test do not depend on the closest t and a child
// rejected early would be rejected later as well (closest only shrinks). The
// sequence of primitive tests, and so the closest-hit result with its
// equal-t tie rule, is the reference's.
//
// Stack: the top `nsh` entries live in shared memory (one column per thread,
// conflict-free), deeper ones in local memory. 32 entries in all; as in the
// reference a push beyond 32 is dropped (and counted). The shared depth is a
// per-scene tunable (SceneView::short_stack, the autotuner's knob, RB_SHORT by
// default); each kernel clamps it to the dynamic shared memory its launch was
// given (stack_init), so a launch can never index past its allocation.
#ifndef RB_SHORT
#define RB_SHORT 8
#endif
#define RB_SHORT_MAX 16
#define RB_STACK 32

struct Stack {
  int2 *sh;     // shared column base for this thread; stride = threads per block
  int stride;
  int nsh;      // entries kept in shared memory
  int2 loc[RB_STACK];
  int sp;
  __device__ __forceinline__ void push(int ref, float te) {
    const int2 e = make_int2(ref, __float_as_int(te));
    if (sp < nsh) sh[sp * stride] = e;
    else loc[sp - nsh] = e;
    ++sp;
  }
  __device__ __forceinline__ int2 pop() {
    --sp;
    return sp < nsh ? sh[sp * stride] : loc[sp - nsh];
  }
};

// Dynamic shared memory of the running launch (PTX special register).
__device__ __forceinline__ unsigned dynamic_smem_bytes() {
  unsigned b;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(b));
  return b;
}

// The stack of thread `tid` of a block of `threads`: `want` shared entries
// (0: RB_SHORT), at most what the launch's dynamic shared memory holds for
// every thread of the block.
__device__ __forceinline__ void stack_init(Stack &st, int2 *smem, int tid, int threads, int want) {
  st.sh = smem + tid;
  st.stride = threads;
  const int cap = (int)(dynamic_smem_bytes() / (sizeof(int2) * (unsigned)threads));
  const int w = want > 0 ? want : RB_SHORT;
  st.nsh = w < cap ? w : cap;
  st.sp = 0;
}

// Dynamic shared memory a launch of `threads` threads provides for a stack of
// `short_stack` shared entries (0: RB_SHORT).
__host__ __device__ inline size_t stack_smem_bytes(int short_stack, int threads) {
  const int w = short_stack > 0 ? (short_stack < RB_SHORT_MAX ? short_stack : RB_SHORT_MAX) : RB_SHORT;
  return sizeof(int2) * (size_t)w * (size_t)threads;
}

struct HitInfo {
  float t;
  int prim;      // primitive, -1 miss, -2 the smooth SDF field
  f3 sdf_n;      // field hit: outward normal and material
  int sdf_mat;
};

// Both child boxes of quantised node `cur` tested against the ray (two
// 128-bit loads from one 32-byte sector); f3v = (left, right, split axis).
// Each bound decodes as corner + q * step in one rounding (q * step is exact).
__device__ __forceinline__ void qnode_visit(const SceneView &S, const RayPre &rp, int cur, float tmin, float closest,
                                            bool &hl, float &tl, bool &hr, float &tr, int4 &f3v) {
  const uint4 *n = reinterpret_cast<const uint4 *>(S.qnodes + cur);
  const uint4 a = __ldg(n), b = __ldg(n + 1);  // (ox, oy, oz, lq0), (lq1, rq, left, right)
  const float ox = qnode_origin(a.x), oy = qnode_origin(a.y), oz = qnode_origin(a.z);
  const float sx = qnode_step(a.x), sy = qnode_step(a.y), sz = qnode_step(a.z);
#define RB_DQ(word, sh, o, s) fmaf((float)(((word) >> (sh)) & 0xFFu), (s), (o))
  hl = box_hit(rp, RB_DQ(a.w, 0, ox, sx), RB_DQ(a.w, 8, oy, sy), RB_DQ(a.w, 16, oz, sz), RB_DQ(a.w, 24, ox, sx),
               RB_DQ(b.x, 0, oy, sy), RB_DQ(b.x, 8, oz, sz), tmin, closest, tl);
  hr = box_hit(rp, RB_DQ(b.x, 16, ox, sx), RB_DQ(b.x, 24, oy, sy), RB_DQ(b.y, 0, oz, sz), RB_DQ(b.y, 8, ox, sx),
               RB_DQ(b.y, 16, oy, sy), RB_DQ(b.y, 24, oz, sz), tmin, closest, tr);
#undef RB_DQ
  f3v = make_int4((int)b.z, (int)b.w, (int)((a.x & 1u) | ((a.y & 1u) << 1)), 0);
}

// Node layout a traversal reads. RB_NODES_ANY decides per scene at run time
// (the 4-wide copy when SceneView::wnodes is set); RB_NODES_BINARY and
// RB_NODES_WIDE fix it at compile time, so that a kernel specialised for one
// layout carries neither the other's code nor its register pressure (the
// wide visit holds 112 B of node words at once: compiled into the diffuse
// class's per-pixel kernel it raised the spills around the traversal from 156
// to 280 bytes per thread, and Cornell, which never runs it, lost 4 %). A
// kernel specialised for RB_NODES_WIDE runs only on scenes that have wnodes.
enum { RB_NODES_ANY = 0, RB_NODES_BINARY = 1, RB_NODES_WIDE = 2 };

static __device__ bool sdf_field_march(const SceneView &S, const Ray &r, float tmin, float tmax, SdfCand &c,
                                       float &t, f3 &n, int &mat);

// Closest hit in [tmin, tmax]. ANY: stop at the first hit (shadow rays).
template <bool ANY, int MS, bool SPEC, class Sink = SdfCand, int NODES = RB_NODES_ANY>
__device__ __forceinline__ HitInfo trace_bvh(const SceneView &S, const Ray &ray, float tmin, float tmax, Stack &st,
                                             uint32_t &overflow, Sink *cand);

// Closest (or, with ANY, first) hit including the smooth SDF field. SPEC
// selects the speculative while-while traversal (render kernels); without it
// the traversal visits nodes and primitives in the reference's exact order.
// RB_SPEC_TRAVERSAL is the render kernels' choice (build with
// -DRB_SPEC_TRAVERSAL=0 for exact-order traversal everywhere).
#ifndef RB_SPEC_TRAVERSAL
#define RB_SPEC_TRAVERSAL 1
#endif
template <bool ANY, int MS, bool SPEC = false, int NODES = RB_NODES_ANY>
__device__ __forceinline__ HitInfo trace(const SceneView &S, const Ray &ray, float tmin, float tmax, Stack &st,
                                         uint32_t &overflow) {
  if (MS >= 4 && S.sdf_k > 0.0f && S.num_sdf > 0) {
    SdfCand cand;
    cand.n = 0;
    HitInfo h = trace_bvh<ANY, MS, SPEC, SdfCand, NODES>(S, ray, tmin, tmax, st, overflow, &cand);
    if (ANY && h.prim >= 0) return h;
    if (cand.n > 0) {
      float ts;
      f3 n;
      int mat;
      if (sdf_field_march(S, ray, tmin, h.t, cand, ts, n, mat)) {
        h.t = ts;
        h.prim = -2;
        h.sdf_n = n;
        h.sdf_mat = mat;
      }
    }
    return h;
  }
  return trace_bvh<ANY, MS, SPEC, SdfCand, NODES>(S, ray, tmin, tmax, st, overflow, static_cast<SdfCand *>(nullptr));
}

template <bool ANY, int MS, class Sink, int NODES>
__device__ __forceinline__ HitInfo trace_ww(const SceneView &S, const Ray &ray, float tmin, float tmax, Stack &st,
                                            uint32_t &overflow, Sink *cand);

template <bool ANY, int MS, bool SPEC, class Sink, int NODES>
__device__ __forceinline__ HitInfo trace_bvh(const SceneView &S, const Ray &ray, float tmin, float tmax, Stack &st,
                                             uint32_t &overflow, Sink *cand) {
  if (SPEC && S.use_bvh) return trace_ww<ANY, MS, Sink, NODES>(S, ray, tmin, tmax, st, overflow, cand);
  HitInfo h;
  h.t = tmax;
  h.prim = -1;
  float closest = tmax;
  if (S.num_groups > 0) {
    // grouped linear layout: groups in leaf order; a group's primitives are
    // tested (in index order, as by the linear scan) when its box is entered
    // before the closest hit
    const RayPre rp = prep(ray);
    for (int gi = 0; gi < S.num_groups; ++gi) {
      const float4 g0 = __ldg(S.groups + 2 * gi), g1 = __ldg(S.groups + 2 * gi + 1);
      float te;
      if (!box_hit(rp, g0.x, g0.y, g0.z, g1.x, g1.y, g1.z, tmin, closest, te)) continue;
      const int first = __float_as_int(g0.w), end = first + __float_as_int(g1.w);
      for (int i = first; i < end; ++i) {
        float t;
        if (prim_t<MS, Sink>(S, i, ray, tmin, closest, t, cand)) {
          closest = t;
          h.t = t;
          h.prim = i;
          if (ANY) return h;
        }
      }
    }
    return h;
  }
  if (!S.use_bvh) {
    for (int i = 0; i < S.num_prims; ++i) {
      float t;
      if (prim_t<MS, Sink>(S, i, ray, tmin, closest, t, cand)) {
        closest = t;
        h.t = t;
        h.prim = i;
        if (ANY) return h;
      }
    }
    return h;
  }
  const RayPre rp = prep(ray);
  float te;
  if (!box_hit(rp, S.root_box[0], S.root_box[1], S.root_box[2], S.root_box[3], S.root_box[4], S.root_box[5], tmin,
               closest, te))
    return h;
  int cur = S.root_ref;
  st.sp = 0;
  int budget = traversal_budget(S);  // bounds a corrupt tree (see trace_ww)
  while (--budget > 0) {
    if (ref_is_leaf(cur)) {
      const int first = leaf_first(cur), cnt = leaf_count(cur);
      for (int i = 0; i < cnt; ++i) {
        float t;
        if (prim_t<MS, Sink>(S, first + i, ray, tmin, closest, t, cand)) {
          closest = t;
          h.t = t;
          h.prim = first + i;
          if (ANY) return h;
        }
      }
    } else {
      float tl, tr;
      bool hl, hr;
      int4 f3v;
      if (!S.quantized) {
        const float4 *n = S.nodes + 4 * (size_t)cur;
        const float4 f0 = __ldg(n), f1 = __ldg(n + 1), f2 = __ldg(n + 2);
        f3v = __ldg(reinterpret_cast<const int4 *>(n + 3));
        hl = box_hit(rp, f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, tmin, closest, tl);
        hr = box_hit(rp, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w, tmin, closest, tr);
      } else {
        qnode_visit(S, rp, cur, tmin, closest, hl, tl, hr, tr, f3v);
      }
      const float dcomp = f3v.z == 0 ? ray.d.x : (f3v.z == 1 ? ray.d.y : ray.d.z);
      const bool left_near = dcomp >= 0.0f;
      const int nref = left_near ? f3v.x : f3v.y, fref = left_near ? f3v.y : f3v.x;
      const bool hn = left_near ? hl : hr, hf = left_near ? hr : hl;
      const float tf = left_near ? tr : tl;
      if (hn) {
        if (hf) {
          if (st.sp < RB_STACK) st.push(fref, tf);
          else ++overflow;
        }
        cur = nref;
        continue;
      }
      if (hf) {
        cur = fref;
        continue;
      }
    }
    // pop the next node whose entry distance still beats the closest hit
    bool found = false;
    while (st.sp > 0) {
      const int2 e = st.pop();
      if (__int_as_float(e.y) <= closest) {
        cur = e.x;
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  note_budget_exhausted(S, budget);
  return h;
}

// Speculative while-while traversal (Aila & Laine, "Understanding the
// Efficiency of Ray Traversal on GPUs", HPG 2009) for the render kernels:
// a lane that reaches a leaf postpones it and keeps visiting interior nodes
// until every still-traversing lane of its warp holds a leaf, then the warp
// tests its leaves together, so interior-node and primitive code run with
// full warps instead of alternating per iteration. Leaves are tested in the
// same front-to-back order; postponing only makes culling by the closest hit
// less eager, so a hit can differ from the exact-order traversal only where a
// primitive test and its box test disagree by a rounding step. A scene
// uploaded with a 4-wide copy of its tree (SceneView::wnodes) is traversed on
// that copy: the same child boxes and leaves, four per visit (visit_wide).
#define RB_TRAV_DONE 0x7FFFFFFF

__device__ __forceinline__ void visit_interior(const SceneView &S, const RayPre &rp, const Ray &ray, int cur, float tmin,
                                               float closest, int &next, Stack &st, uint32_t &overflow) {
  float tl, tr;
  bool hl, hr;
  int4 f3v;
  if (!S.quantized) {
    const float4 *n = S.nodes + 4 * (size_t)cur;
    const float4 f0 = __ldg(n), f1 = __ldg(n + 1), f2 = __ldg(n + 2);
    f3v = __ldg(reinterpret_cast<const int4 *>(n + 3));
    hl = box_hit(rp, f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, tmin, closest, tl);
    hr = box_hit(rp, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w, tmin, closest, tr);
  } else {
    qnode_visit(S, rp, cur, tmin, closest, hl, tl, hr, tr, f3v);
  }
  const float dcomp = f3v.z == 0 ? ray.d.x : (f3v.z == 1 ? ray.d.y : ray.d.z);
  const bool left_near = dcomp >= 0.0f;
  const int nref = left_near ? f3v.x : f3v.y, fref = left_near ? f3v.y : f3v.x;
  const bool hn = left_near ? hl : hr, hf = left_near ? hr : hl;
  const float tf = left_near ? tr : tl;
  if (hn) {
    if (hf) {
      if (st.sp < RB_STACK) st.push(fref, tf);
      else ++overflow;
    }
    next = nref;
  } else if (hf) {
    next = fref;
  } else {
    next = RB_TRAV_DONE;  // pop below
  }
}

// One 4-wide node (wide_bvh.cu: 128 B, bounds of the four children in the
// lanes of six words, then the child refs): the hit children are ordered by
// entry distance with a five-exchange sorting network, the farther ones pushed
// from far to near so that the nearest pending child is popped first, and the
// nearest becomes `next`.
__device__ __forceinline__ void visit_wide(const SceneView &S, const RayPre &rp, int cur, float tmin, float closest,
                                           int &next, Stack &st, uint32_t &overflow) {
  const float4 *n = S.wnodes + 8 * (size_t)cur;
  const float4 lx = __ldg(n), hx = __ldg(n + 1), ly = __ldg(n + 2), hy = __ldg(n + 3), lz = __ldg(n + 4),
               hz = __ldg(n + 5);
  const int4 rf = __ldg(reinterpret_cast<const int4 *>(n + 6));
  const float INF = __int_as_float(0x7f800000);
  float k0, k1, k2, k3;
  int r0 = rf.x, r1 = rf.y, r2 = rf.z, r3 = rf.w;
  k0 = box_hit(rp, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, tmin, closest, k0) ? k0 : INF;
  k1 = box_hit(rp, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, tmin, closest, k1) ? k1 : INF;
  k2 = box_hit(rp, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, tmin, closest, k2) ? k2 : INF;
  k3 = box_hit(rp, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, tmin, closest, k3) ? k3 : INF;
#define RB_CX(a, b)                                       \
  if (k##b < k##a) {                                      \
    const float tk = k##a; k##a = k##b; k##b = tk;        \
    const int tr = r##a; r##a = r##b; r##b = tr;          \
  }
  RB_CX(0, 1) RB_CX(2, 3) RB_CX(0, 2) RB_CX(1, 3) RB_CX(1, 2)
#undef RB_CX
#define RB_PUSH_W(k, r)                     \
  if (k < INF) {                            \
    if (st.sp < RB_STACK) st.push(r, k);    \
    else ++overflow;                        \
  }
  RB_PUSH_W(k3, r3) RB_PUSH_W(k2, r2) RB_PUSH_W(k1, r1)
#undef RB_PUSH_W
  next = k0 < INF ? r0 : RB_TRAV_DONE;
}

__device__ __forceinline__ int pop_next(Stack &st, float closest) {
  while (st.sp > 0) {
    const int2 e = st.pop();
    if (__int_as_float(e.y) <= closest) return e.x;
  }
  return RB_TRAV_DONE;
}

template <bool ANY, int MS, class Sink, int NODES>
__device__ __forceinline__ HitInfo trace_ww(const SceneView &S, const Ray &ray, float tmin, float tmax, Stack &st,
                                            uint32_t &overflow, Sink *cand) {
  HitInfo h;
  h.t = tmax;
  h.prim = -1;
  float closest = tmax;
  const RayPre rp = prep(ray);
  float te;
  if (!box_hit(rp, S.root_box[0], S.root_box[1], S.root_box[2], S.root_box[3], S.root_box[4], S.root_box[5], tmin,
               closest, te))
    return h;
  st.sp = 0;
  const bool wide = NODES == RB_NODES_WIDE || (NODES == RB_NODES_ANY && S.wnodes != nullptr);
  int node = wide ? S.wide_root : S.root_ref;
  int leaf = RB_TRAV_DONE;  // postponed leaf
  // every interior node and every leaf is visited at most once, so this
  // budget is never reached by a well-formed tree; it bounds a corrupt one
  int budget = traversal_budget(S);
  while ((node != RB_TRAV_DONE || leaf != RB_TRAV_DONE) && --budget > 0) {
    // interior phase
    while (node != RB_TRAV_DONE && !ref_is_leaf(node) && --budget > 0) {
      int next;
      if (wide) visit_wide(S, rp, node, tmin, closest, next, st, overflow);
      else visit_interior(S, rp, ray, node, tmin, closest, next, st, overflow);
      node = next == RB_TRAV_DONE ? pop_next(st, closest) : next;
      if (node != RB_TRAV_DONE && ref_is_leaf(node) && leaf == RB_TRAV_DONE) {
        leaf = node;  // postpone and keep descending
        node = pop_next(st, closest);
      }
      if (__all_sync(__activemask(), leaf != RB_TRAV_DONE)) break;
    }
    // a leaf reached without a postponed one (e.g. the root is a leaf)
    if (leaf == RB_TRAV_DONE && node != RB_TRAV_DONE && ref_is_leaf(node)) {
      leaf = node;
      node = pop_next(st, closest);
    }
    // leaf phase: the postponed leaf, then `node` if it is one too
    while (leaf != RB_TRAV_DONE) {
      const int first = leaf_first(leaf), cnt = leaf_count(leaf);
      for (int i = 0; i < cnt; ++i) {
        float t;
        if (prim_t<MS, Sink>(S, first + i, ray, tmin, closest, t, cand)) {
          closest = t;
          h.t = t;
          h.prim = first + i;
          if (ANY) return h;
        }
      }
      leaf = RB_TRAV_DONE;
      if (node != RB_TRAV_DONE && ref_is_leaf(node)) {
        leaf = node;
        node = pop_next(st, closest);
      }
    }
  }
  note_budget_exhausted(S, budget);
  return h;
}

// ---------------------------------------------------------------------------
// Surface at the closest hit (hit record fields of cuda_raytracer.cuh:203-347)
// ---------------------------------------------------------------------------
struct Surface {
  f3 p, n, tangent, center;
  bool front;
  bool visible;
  int mat;
};

static __device__ Surface golf_surface(const f3 &center, float radius, const Ray &r, float t);
static __device__ Surface sdf_surface(const SceneView &S, int prim, const Ray &r, float t);

template <int MS>
__device__ __forceinline__ Surface surface(const SceneView &S, const Ray &r, const HitInfo &h) {
  if (MS >= 4 && h.prim == -2) {  // smooth SDF field; the point is lifted 4 eps off the surface
    Surface s;
    s.p = r.at(h.t) + (4.0f * S.sdf_eps) * h.sdf_n * (dot(r.d, h.sdf_n) < 0 ? 1.0f : -1.0f);
    s.front = dot(r.d, h.sdf_n) < 0;
    s.n = s.front ? h.sdf_n : f3(-h.sdf_n.x, -h.sdf_n.y, -h.sdf_n.z);
    f3 tg = cross(f3(0.0f, 1.0f, 0.0f), h.sdf_n);
    if (tg.length_squared() < 1e-6f) tg = f3(1.0f, 0.0f, 0.0f);
    s.tangent = normalize(tg);
    s.center = f3(0.0f, 0.0f, 0.0f);
    s.visible = true;
    s.mat = h.sdf_mat;
    return s;
  }
  const float4 *p = S.prims + 3 * (size_t)h.prim;
  const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  const uint32_t tag = __float_as_uint(c.w);
  const uint32_t kind = tag_kind(tag);
  Surface s;
  s.visible = tag_visible(tag);
  s.mat = tag_material(tag);
  s.center = f3(0.0f, 0.0f, 0.0f);
  if (kind == PK_SPHERE) {
    const f3 center(a.x, a.y, a.z);
    const float radius = a.w;
    s.p = r.at(h.t);
    f3 outward = (s.p - center) / radius;
    s.front = dot(r.d, outward) < 0;
    s.n = s.front ? outward : f3(-outward.x, -outward.y, -outward.z);
    f3 tg = cross(f3(0.0f, 1.0f, 0.0f), outward);
    if (tg.length_squared() < 1e-6f) tg = f3(1.0f, 0.0f, 0.0f);
    s.tangent = normalize(tg);
    s.center = center;
  } else if (kind == PK_RECT) {
    const f3 u(a.w, b.x, b.y), v(b.z, b.w, c.x);
    f3 normal = normalize(f3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x));
    s.p = r.at(h.t);
    s.front = dot(r.d, normal) < 0;
    s.n = s.front ? normal : f3(-normal.x, -normal.y, -normal.z);
    s.tangent = normalize(u);
  } else if (kind == PK_TRI) {
    const f3 v0(a.x, a.y, a.z), e1(a.w, b.x, b.y), e2(b.z, b.w, c.x);
    s.p = r.at(h.t);
    const f3 geo = normalize(cross(e1, e2));
    s.front = dot(r.d, geo) < 0;
    f3 sn = geo;
    const bool has_n = tag_normals(tag) && S.normals != nullptr;
    if (has_n) {
      const f3 hh = cross(r.d, e2);
      const float f = 1.0f / dot(e1, hh);
      const f3 sv = r.o - v0;
      const float uu = f * dot(sv, hh);
      const f3 q = cross(sv, e1);
      const float vv = f * dot(r.d, q);
      const float w = 1.0f - uu - vv;
      const float4 *np = S.normals + 3 * (size_t)h.prim;
      const f3 n0 = mk(__ldg(np)), n1 = mk(__ldg(np + 1)), n2 = mk(__ldg(np + 2));
      sn = normalize(w * n0 + uu * n1 + vv * n2);
      if (dot(sn, geo) < 0.0f) sn = -sn;
    }
    s.n = s.front ? sn : -sn;
    if (has_n) {
      const f3 incoming = -r.d;
      if (dot(s.n, incoming) <= 0.0f) s.n = s.front ? geo : -geo;
    }
    s.tangent = normalize(e1);
  } else if (MS >= 3 && kind == PK_DISPLACED) {
    Surface g = golf_surface(f3(a.x, a.y, a.z), a.w, r, h.t);
    g.visible = s.visible;
    g.mat = s.mat;
    return g;
  } else if (MS >= 4) {
    Surface g = sdf_surface(S, h.prim, r, h.t);
    g.visible = s.visible;
    g.mat = s.mat;
    return g;
  }
  return s;
}

}  // namespace rbd
