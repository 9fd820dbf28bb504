// 8-bit quantised BVH nodes with outward rounding.
//
// Each interior node stores its children's boxes on a per-axis power-of-two
// grid anchored at the union box's minimum corner. Decoding on the device is
// origin + q * 2^e in FP32; q * 2^e is exact, so the decoded bound is one
// rounded addition, which this file evaluates the same way and nudges q until
// min bounds decode <= the FP32 bound and max bounds decode >= it. The decoded
// box therefore contains the FP32 box, and because rounded subtraction and
// multiplication are monotone, the slab test on it accepts every ray the FP32
// box accepts with an entry distance no larger.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "rb_internal.hpp"

namespace rb {

namespace {

float decode(float origin, int q, float scale) {
  volatile float prod = (float)q * scale;  // exact: q < 256, scale a power of two
  volatile float sum = origin + prod;      // one rounding, as on the device
  return sum;
}

int exponent_for(float extent) {
  // smallest e with 255 * 2^e >= extent (biased exponent byte, 1..254)
  if (!(extent > 0.0f)) return 1;
  int e = (int)std::ceil(std::log2((double)extent / 255.0));
  while (std::ldexp(255.0, e) < (double)extent) ++e;
  int biased = e + 127;
  if (biased < 1) biased = 1;
  if (biased > 254) biased = 254;
  return biased;
}

float scale_of(int biased) {
  uint32_t bits = (uint32_t)biased << 23;
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

}  // namespace

void build_quantized(HostLayout &L) {
  const size_t n = L.nodes.size() / 4;
  L.qnodes.assign(n, rbd::QNode());
  for (size_t i = 0; i < n; ++i) {
    const float *w = reinterpret_cast<const float *>(&L.nodes[4 * i]);
    const int *wi = reinterpret_cast<const int *>(&L.nodes[4 * i + 3]);
    float lo[2][3], hi[2][3];
    for (int k = 0; k < 3; ++k) {
      lo[0][k] = w[k]; hi[0][k] = w[3 + k];
      lo[1][k] = w[6 + k]; hi[1][k] = w[9 + k];
    }
    rbd::QNode q;
    std::memset(&q, 0, sizeof q);
    float origin[3];
    int ex[3];
    float sc[3];
    for (int k = 0; k < 3; ++k) {
      origin[k] = std::fmin(lo[0][k], lo[1][k]);
      const float top = std::fmax(hi[0][k], hi[1][k]);
      ex[k] = exponent_for((float)((double)top - (double)origin[k]) * 1.0001f);
      sc[k] = scale_of(ex[k]);
      // make sure the whole range is reachable after rounding
      while (decode(origin[k], 255, sc[k]) < top && ex[k] < 254) sc[k] = scale_of(++ex[k]);
    }
    q.ox = origin[0]; q.oy = origin[1]; q.oz = origin[2];
    q.meta = (uint32_t)ex[0] | ((uint32_t)ex[1] << 8) | ((uint32_t)ex[2] << 16) | ((uint32_t)wi[2] << 24);
    uint8_t b[2][6];
    for (int c = 0; c < 2; ++c)
      for (int k = 0; k < 3; ++k) {
        int ql = (int)std::floor(((double)lo[c][k] - (double)origin[k]) / (double)sc[k]);
        ql = ql < 0 ? 0 : (ql > 255 ? 255 : ql);
        while (ql > 0 && decode(origin[k], ql, sc[k]) > lo[c][k]) --ql;
        int qh = (int)std::ceil(((double)hi[c][k] - (double)origin[k]) / (double)sc[k]);
        qh = qh < 0 ? 0 : (qh > 255 ? 255 : qh);
        while (qh < 255 && decode(origin[k], qh, sc[k]) < hi[c][k]) ++qh;
        b[c][k] = (uint8_t)ql;
        b[c][3 + k] = (uint8_t)qh;
      }
    // L: lo x y z, hi x | hi y z, R lo x y | R lo z, hi x y z
    q.lq0 = b[0][0] | (b[0][1] << 8) | (b[0][2] << 16) | ((uint32_t)b[0][3] << 24);
    q.lq1 = b[0][4] | (b[0][5] << 8) | (b[1][0] << 16) | ((uint32_t)b[1][1] << 24);
    q.rq = b[1][2] | (b[1][3] << 8) | (b[1][4] << 16) | ((uint32_t)b[1][5] << 24);
    q.left = wi[0];
    q.right = wi[1];
    L.qnodes[i] = q;
  }
}

}  // namespace rb
