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
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <deque>
#include <limits>
#include <thread>
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

// The up-to-four children of the wide node that replaces binary interior
// node `bref`: its two children, then the interior child of largest surface
// area opened until four are held or only leaves remain.
int collapse(const HostLayout &L, int bref, Child ch[4]) {
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
  return n;
}

// Writes one wide node (8 words) with child refs `refs` (interior children
// get their ref patched later where it is not known yet).
void write_node(float4 *dst, const Child ch[4], int n, const int refs[4]) {
  const float inf = std::numeric_limits<float>::infinity();
  float *w = reinterpret_cast<float *>(dst);
  for (int c = 0; c < 4; ++c)
    for (int k = 0; k < 3; ++k) {
      w[8 * k + c] = c < n ? ch[c].lo[k] : inf;
      w[8 * k + 4 + c] = c < n ? ch[c].hi[k] : inf;
    }
  int *wi = reinterpret_cast<int *>(dst + 6);
  for (int c = 0; c < 4; ++c) wi[c] = refs[c];
  for (int c = 4; c < 8; ++c) wi[c] = 0;
}

int *ref_slot(float4 *node, int lane) { return reinterpret_cast<int *>(node + 6) + lane; }

// The wide subtree of binary interior node `bref` in depth-first order, its
// root at local slot 0 and interior refs local to `out`.
void build_subtree(const HostLayout &L, int bref, std::vector<float4> &out) {
  std::vector<std::pair<int, int>> todo{{bref, 0}};
  out.resize(8);
  while (!todo.empty()) {
    const auto [b, slot] = todo.back();
    todo.pop_back();
    Child ch[4];
    const int n = collapse(L, b, ch);
    int refs[4] = {0, 0, 0, 0};
    for (int c = 0; c < n; ++c) {
      if (rbd::ref_is_leaf(ch[c].ref)) {
        refs[c] = ch[c].ref;
      } else {
        refs[c] = (int)(out.size() / 8);  // children of a node sit next to each other
        out.resize(out.size() + 8);
        todo.push_back({ch[c].ref, refs[c]});
      }
    }
    write_node(&out[8 * (size_t)slot], ch, n, refs);
  }
}

}  // namespace

// The top of the tree is collapsed breadth-first on one thread until it has
// at least 256 pending interior children; their subtrees are then built on
// all host cores (each a depth-first block) and appended in order, their
// interior refs shifted to the block's position (the nodes reached through
// one top-level child stay contiguous, as in a single depth-first build).
void build_wide(HostLayout &L) {
  L.wnodes.clear();
  L.wide_root = L.root_ref;
  if (!L.use_bvh || L.nodes.empty() || rbd::ref_is_leaf(L.root_ref)) return;
  struct Pending {
    int bref, parent, lane;
  };
  std::vector<float4> top;
  std::deque<Pending> q;
  auto emit = [&](int bref) {
    const int slot = (int)(top.size() / 8);
    top.resize(top.size() + 8);
    Child ch[4];
    const int n = collapse(L, bref, ch);
    int refs[4] = {0, 0, 0, 0};
    for (int c = 0; c < n; ++c) {
      if (rbd::ref_is_leaf(ch[c].ref)) refs[c] = ch[c].ref;
      else q.push_back({ch[c].ref, slot, c});
    }
    write_node(&top[8 * (size_t)slot], ch, n, refs);
    return slot;
  };
  L.wide_root = emit(L.root_ref);  // slot 0
  while (!q.empty() && q.size() < 256) {
    const Pending p = q.front();
    q.pop_front();
    const int slot = emit(p.bref);
    *ref_slot(&top[8 * (size_t)p.parent], p.lane) = slot;
  }
  const std::vector<Pending> rest(q.begin(), q.end());
  std::vector<std::vector<float4>> sub(rest.size());
  {
    const size_t threads = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 64);
    std::atomic<size_t> next{0};
    auto work = [&]() {
      for (size_t i = next++; i < rest.size(); i = next++) build_subtree(L, rest[i].bref, sub[i]);
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < threads && t < rest.size(); ++t) pool.emplace_back(work);
    work();
    for (auto &th : pool) th.join();
  }
  std::vector<size_t> base(rest.size());
  size_t total = top.size();
  for (size_t i = 0; i < rest.size(); ++i) {
    base[i] = total / 8;
    total += sub[i].size();
  }
  L.wnodes.resize(total);
  std::copy(top.begin(), top.end(), L.wnodes.begin());
  for (size_t i = 0; i < rest.size(); ++i) {
    *ref_slot(&L.wnodes[8 * (size_t)rest[i].parent], rest[i].lane) = (int)base[i];
    float4 *dst = &L.wnodes[8 * base[i]];
    std::copy(sub[i].begin(), sub[i].end(), dst);
    const int shift = (int)base[i];
    for (size_t k = 0; k < sub[i].size() / 8; ++k) {
      const float *w = reinterpret_cast<const float *>(dst + 8 * k);
      int *refs = reinterpret_cast<int *>(dst + 8 * k + 6);
      for (int c = 0; c < 4; ++c)  // valid interior children: a finite bound, a non-leaf ref
        if (std::isfinite(w[c]) && !rbd::ref_is_leaf(refs[c])) refs[c] += shift;
    }
  }
}

}  // namespace rb
