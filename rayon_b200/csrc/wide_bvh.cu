// 4-wide copy of the binary BVH for the render kernels' traversal.
//
// Each wide node is the binary tree collapsed two levels at a time: starting
// from a binary node's two children, the interior child with the largest box
// surface area is replaced by its own two children until the node holds four
// children or only leaves remain. The child boxes and leaf references are the
// binary tree's own (FP32, unchanged), so the wide tree bounds exactly the same
// primitive ranges; a visit tests up to four boxes from one 128-byte line, and
// a ray descends about half as many levels, so the chain of dependent node
// loads that bounds incoherent traversal is about half as long.
//
// Node layout (8 x float4 = 128 B): lo.x[4], hi.x[4], lo.y[4], hi.y[4],
// lo.z[4], hi.z[4] (child c in lane c of each word), then the four child refs
// (interior: wide node index; leaf: the binary tree's leaf encoding) and a
// padding word. An empty child slot has every bound at +inf, which the slab
// test rejects for every ray (both slab distances are +inf or both -inf).
#include <cmath>
#include <cstring>
#include <limits>
#include <utility>
#include <vector>

#include "rb_internal.hpp"

namespace rb {

namespace {

struct Child {
  int ref;
  float lo[3], hi[3];
};

float area(const Child &c) {
  const float dx = c.hi[0] - c.lo[0], dy = c.hi[1] - c.lo[1], dz = c.hi[2] - c.lo[2];
  return dx * dy + dy * dz + dz * dx;
}

// The two children of binary interior node `ref` (L.nodes, 4 words each).
void binary_children(const HostLayout &L, int ref, Child out[2]) {
  const float *w = reinterpret_cast<const float *>(&L.nodes[4 * (size_t)ref]);
  const int *wi = reinterpret_cast<const int *>(&L.nodes[4 * (size_t)ref + 3]);
  for (int k = 0; k < 3; ++k) {
    out[0].lo[k] = w[k];
    out[0].hi[k] = w[3 + k];
    out[1].lo[k] = w[6 + k];
    out[1].hi[k] = w[9 + k];
  }
  out[0].ref = wi[0];
  out[1].ref = wi[1];
}

}  // namespace

void build_wide(HostLayout &L) {
  L.wnodes.clear();
  L.wide_root = L.root_ref;
  if (!L.use_bvh || L.nodes.empty() || rbd::ref_is_leaf(L.root_ref)) return;
  const size_t nbin = L.nodes.size() / 4;
  L.wnodes.reserve(8 * (nbin / 2 + 1));
  const float inf = std::numeric_limits<float>::infinity();
  auto alloc = [&]() {
    const int slot = (int)(L.wnodes.size() / 8);
    L.wnodes.resize(L.wnodes.size() + 8);
    return slot;
  };
  std::vector<std::pair<int, int>> todo;  // (binary interior ref, wide slot)
  L.wide_root = alloc();
  todo.push_back({L.root_ref, L.wide_root});
  while (!todo.empty()) {
    const auto [bref, slot] = todo.back();
    todo.pop_back();
    Child ch[4];
    int n = 2;
    binary_children(L, bref, ch);
    while (n < 4) {
      int best = -1;
      float best_area = -1.0f;
      for (int c = 0; c < n; ++c)
        if (!rbd::ref_is_leaf(ch[c].ref) && area(ch[c]) > best_area) {
          best = c;
          best_area = area(ch[c]);
        }
      if (best < 0) break;
      Child two[2];
      binary_children(L, ch[best].ref, two);
      ch[best] = two[0];
      ch[n++] = two[1];
    }
    int refs[4] = {0, 0, 0, 0};
    for (int c = 0; c < n; ++c) {
      if (rbd::ref_is_leaf(ch[c].ref)) {
        refs[c] = ch[c].ref;
      } else {
        refs[c] = alloc();  // children of a node sit next to each other
        todo.push_back({ch[c].ref, refs[c]});
      }
    }
    float *w = reinterpret_cast<float *>(&L.wnodes[8 * (size_t)slot]);
    for (int c = 0; c < 4; ++c)
      for (int k = 0; k < 3; ++k) {
        w[8 * k + c] = c < n ? ch[c].lo[k] : inf;
        w[8 * k + 4 + c] = c < n ? ch[c].hi[k] : inf;
      }
    int *wi = reinterpret_cast<int *>(&L.wnodes[8 * (size_t)slot + 6]);
    for (int c = 0; c < 4; ++c) wi[c] = refs[c];
    for (int c = 4; c < 8; ++c) wi[c] = 0;
  }
}

}  // namespace rb
