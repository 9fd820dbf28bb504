/* Counter-based random numbers shared by the CUDA kernels and the CPU oracle.
 *
 * Every random number of a path is a pure function of
 * (seed, job salt, pixel, sample, dimension): a path's key is a hash of the
 * first four, and draw `dim` is hash(key + dim * golden). Nothing is carried
 * between draws, so a path gives the same numbers whichever kernel, launch
 * shape, batch or job mix runs it, and the CPU oracle reproduces them bit for
 * bit. The 24-bit float mapping is exact in FP32 and FP64.
 *
 * The mixing function is the "lowbias32" integer hash (Chris Wellons,
 * hash-prospector, public domain): xorshift-multiply rounds with constants
 * 0x7feb352d and 0x846ca68b.
 *
 * Dimension layout of one path (fixed slots, so a branch taken differently at
 * one vertex does not shift the numbers used at later vertices):
 *   0-1 pixel jitter, 2-3 lens sample,
 *   RB_DIM_VERTEX0 + RB_DIM_PER_VERTEX * bounce + slot, slot:
 *     0-1 BSDF direction, 2 lobe choice, 3-4 secondary lobe direction,
 *     5 Russian roulette, 6 light choice, 7-8 point on light.
 */
#ifndef RB_RNG_H
#define RB_RNG_H

#include <stdint.h>

#if defined(__CUDACC__)
#define RB_HD __host__ __device__ __forceinline__
#else
#define RB_HD static inline
#endif

#define RB_DIM_JITTER 0
#define RB_DIM_LENS 2
#define RB_DIM_VERTEX0 4
#define RB_DIM_PER_VERTEX 9
#define RB_SLOT_BSDF 0
#define RB_SLOT_LOBE 2
#define RB_SLOT_BSDF2 3
#define RB_SLOT_RR 5
#define RB_SLOT_LIGHT 6
#define RB_SLOT_LIGHT_PT 7

RB_HD uint32_t rb_hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

/* Key of one path. salt distinguishes jobs (0 for the drop-in renderer). */
RB_HD uint32_t rb_path_key(uint32_t seed, uint32_t salt, uint32_t pixel, uint32_t sample) {
  uint32_t h = rb_hash32(sample * 0x9E3779B9U + salt);
  h = rb_hash32(h ^ (pixel * 0x85EBCA6BU + 0x632BE5ABU));
  return rb_hash32(h ^ seed);
}

RB_HD uint32_t rb_draw_u32(uint32_t key, uint32_t dim) {
  return rb_hash32(key + dim * 0x9E3779B9U);
}

/* [0, 1) with 24 bits; exact in float and double. */
RB_HD float rb_draw(uint32_t key, uint32_t dim) {
  return (float)(rb_draw_u32(key, dim) >> 8) * (1.0f / 16777216.0f);
}
RB_HD double rb_draw_d(uint32_t key, uint32_t dim) {
  return (double)(rb_draw_u32(key, dim) >> 8) * (1.0 / 16777216.0);
}

RB_HD uint32_t rb_vdim(int bounce, int slot) {
  return (uint32_t)(RB_DIM_VERTEX0 + RB_DIM_PER_VERTEX * bounce + slot);
}

#endif /* RB_RNG_H */
