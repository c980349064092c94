// Collapse of the reference's binary BVH (BVH_GPU layout, bvh.glsl:1-6) into
// a 4-wide BVH for the device traversal.
//
// A binary node stores the boxes of its two children; a wide node stores the
// boxes of up to four descendants taken from the binary tree: starting from
// the two children of a binary inner node, the inner child with the largest
// box surface area is replaced by its own two children until there are four
// (or only leaves are left).  Every box of the wide tree is therefore a box of
// the binary tree, bit for bit, and a ray/box test of the wide traversal gives
// the same answer as the same test in the binary traversal.  Binary leaves
// become entries of a leaf table holding the clipped range of leaf slots the
// reference would test: [max(first, 0), min(first + min(cnt, 64), slots))
// (bvh.glsl:160-176).  Children the reference would not push (index out of
// range, a node referring to itself) are left out, and a node reached twice
// (a malformed, cyclic input) is expanded once.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bvh_wide.h"

namespace dspbr {

namespace {

struct ChildRef {
  int node;       // binary node index
  float box[6];   // lo.xyz, hi.xyz as stored in the binary parent
};

float surface(const float* b) {
  float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
  if (!(dx >= 0.f) || !(dy >= 0.f) || !(dz >= 0.f)) return 0.f;  // empty / NaN boxes are not expanded first
  return dx * dy + dy * dz + dz * dx;
}

}  // namespace

// nodes: 16 floats per binary node with child / count / first stored as int
// bits in lanes 3, 7, 11, 15 (the device layout of DevScene::nodes).
WideBvh collapse_bvh4(const float* nodes, uint32_t num_nodes, uint32_t num_slots) {
  WideBvh w;
  auto as_int = [](float f) {
    int v;
    std::memcpy(&v, &f, 4);
    return v;
  };
  auto is_leaf = [&](int n) { return as_int(nodes[16 * size_t(n) + 11]) > 0; };
  auto add_leaf = [&](int n) {
    const float* b = nodes + 16 * size_t(n);
    int cnt = as_int(b[11]), first = as_int(b[15]);
    int64_t lo = std::max(first, 0);
    int64_t hi = std::min<int64_t>(int64_t(first) + std::min(cnt, kWideMaxLeafTris), int64_t(num_slots));
    if (hi < lo) hi = lo;
    w.leaves.push_back({int32_t(lo), int32_t(hi)});
    return int32_t(w.leaves.size() - 1);
  };
  if (num_nodes == 0) return w;
  if (is_leaf(0)) {  // the root itself is a leaf: its triangles are tested without a box test
    w.root = ~add_leaf(0);
    return w;
  }
  std::vector<uint8_t> seen(num_nodes, 0);
  struct Pending {
    int binary;  // binary inner node whose children become the wide node's
    int slot;    // wide node index
  };
  std::vector<Pending> work;
  w.nodes.emplace_back();
  work.push_back({0, 0});
  seen[0] = 1;
  w.root = 0;
  while (!work.empty()) {
    Pending pj = work.back();
    work.pop_back();
    // the binary node's two children, as bvh_push_child would push them
    ChildRef kids[4];
    int nk = 0;
    auto children_of = [&](int n, ChildRef* out) {
      const float* b = nodes + 16 * size_t(n);
      int left = as_int(b[3]), right = as_int(b[7]);
      ChildRef cand[2] = {{left, {b[0], b[1], b[2], b[4], b[5], b[6]}},
                          {right, {b[8], b[9], b[10], b[12], b[13], b[14]}}};
      int m = 0;
      for (const ChildRef& c : cand)
        if (c.node >= 0 && uint32_t(c.node) < num_nodes && c.node != n) out[m++] = c;
      return m;
    };
    nk = children_of(pj.binary, kids);
    // open inner children (largest surface first) while there is room
    for (;;) {
      int best = -1;
      float best_area = -1.f;
      ChildRef grand[2];
      for (int k = 0; k < nk; ++k) {
        int n = kids[k].node;
        if (is_leaf(n) || seen[n]) continue;
        if (nk - 1 + children_of(n, grand) > 4) continue;
        float a = surface(kids[k].box);
        if (a > best_area) {
          best_area = a;
          best = k;
        }
      }
      if (best < 0) break;
      int n = kids[best].node;
      seen[n] = 1;
      int ng = children_of(n, grand);
      for (int k = best; k + 1 < nk; ++k) kids[k] = kids[k + 1];
      --nk;
      for (int k = 0; k < ng; ++k) kids[nk++] = grand[k];
    }
    WideNode4 out{};
    for (int k = 0; k < 4; ++k) {
      out.lo_x[k] = out.lo_y[k] = out.lo_z[k] = 0.f;
      out.hi_x[k] = out.hi_y[k] = out.hi_z[k] = 0.f;
      out.child[k] = 0;
    }
    out.count = nk;
    for (int k = 0; k < nk; ++k) {
      const ChildRef& c = kids[k];
      out.lo_x[k] = c.box[0]; out.lo_y[k] = c.box[1]; out.lo_z[k] = c.box[2];
      out.hi_x[k] = c.box[3]; out.hi_y[k] = c.box[4]; out.hi_z[k] = c.box[5];
      if (is_leaf(c.node)) {
        out.child[k] = ~add_leaf(c.node);
      } else if (seen[c.node]) {
        out.child[k] = ~int32_t(w.leaves.size());  // reached twice: an empty leaf
        w.leaves.push_back({0, 0});
      } else {
        seen[c.node] = 1;
        int32_t slot = int32_t(w.nodes.size());
        w.nodes.emplace_back();
        out.child[k] = slot;
        work.push_back({c.node, slot});
      }
    }
    w.nodes[pj.slot] = out;
  }
  return w;
}

}  // namespace dspbr
