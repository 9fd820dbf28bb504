// 8-bit quantised BVH nodes with outward rounding.
//
// Each interior node (32 B, one sector) stores its children's boxes on a
// per-axis power-of-two grid anchored at the union box's minimum corner, the
// corner kept to 24 bits and rounded toward -inf. Decoding on the device is
// corner + q * 2^e in FP32; q * 2^e is exact, so the decoded bound is one
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

uint32_t f2u(float f) {
  uint32_t b;
  std::memcpy(&b, &f, 4);
  return b;
}
float u2f(uint32_t b) {
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

float decode(float origin, int q, float scale) {
  volatile float prod = (float)q * scale;  // exact: q < 256, scale a power of two
  volatile float sum = origin + prod;      // one rounding, as on the device
  return sum;
}

// The grid corner kept in a node: the coordinate's FP32 bits with the low 8
// mantissa bits dropped, rounded toward -inf (never above the coordinate).
float corner_of(float o) {
  uint32_t b = f2u(o);
  if (b & 0xFFu) b = (b & 0x80000000u) ? (b & ~0xFFu) + 0x100u : (b & ~0xFFu);
  return u2f(b);
}

// Step 2^e stored as e + 64 in 7 bits (e in [-64, 63]).
float step_of(int e) { return u2f((uint32_t)(e + 127) << 23); }

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
    float corner[3], sc[3];
    int ex[3];
    for (int k = 0; k < 3; ++k) {
      corner[k] = corner_of(std::fmin(lo[0][k], lo[1][k]));
      const float top = std::fmax(hi[0][k], hi[1][k]);
      const double extent = ((double)top - (double)corner[k]) * 1.0001;
      int e = extent > 0.0 ? (int)std::ceil(std::log2(extent / 255.0)) : -64;
      e = e < -64 ? -64 : (e > 63 ? 63 : e);
      while (e < 63 && std::ldexp(255.0, e) < extent) ++e;
      // make sure the whole range is reachable after rounding
      while (e < 63 && decode(corner[k], 255, step_of(e)) < top) ++e;
      ex[k] = e;
      sc[k] = step_of(e);
    }
    const uint32_t axis = (uint32_t)wi[2] & 3u;
    rbd::QNode q;
    q.ox = (f2u(corner[0]) & 0xFFFFFF00u) | ((uint32_t)(ex[0] + 64) << 1) | (axis & 1u);
    q.oy = (f2u(corner[1]) & 0xFFFFFF00u) | ((uint32_t)(ex[1] + 64) << 1) | (axis >> 1);
    q.oz = (f2u(corner[2]) & 0xFFFFFF00u) | ((uint32_t)(ex[2] + 64) << 1);
    uint8_t b[2][6];
    for (int c = 0; c < 2; ++c)
      for (int k = 0; k < 3; ++k) {
        int ql = (int)std::floor(((double)lo[c][k] - (double)corner[k]) / (double)sc[k]);
        ql = ql < 0 ? 0 : (ql > 255 ? 255 : ql);
        while (ql > 0 && decode(corner[k], ql, sc[k]) > lo[c][k]) --ql;
        int qh = (int)std::ceil(((double)hi[c][k] - (double)corner[k]) / (double)sc[k]);
        qh = qh < 0 ? 0 : (qh > 255 ? 255 : qh);
        while (qh < 255 && decode(corner[k], qh, sc[k]) < hi[c][k]) ++qh;
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
