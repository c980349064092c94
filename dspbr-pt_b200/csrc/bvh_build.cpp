// Binned-SAH BVH builder that emits the reference's binary BVH node layout.
//
// Replaces the TinyBVH WASM builder (packages/lib/bvh/tinybvh_builder.ts:43-256,
// module ABI :7-24), whose source is not part of the reference.  Output format
// is the one the reference's traversal reads (packages/lib/shader/bvh.glsl:1-6):
// 16 floats per node
//     (lmin.xyz, left) (lmax.xyz, right) (rmin.xyz, cnt) (rmax.xyz, first)
// root = node 0, leaf iff cnt > 0, leaf triangles = remap[first .. first+cnt).
// Child indices, counts and offsets are stored as floats (exact below 2^24),
// as in the reference.  Depth is bounded so that the traversal's 64-entry stack
// (bvh.glsl:8) can never overflow on trees built here.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <future>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "dspbr.h"

namespace dspbr {
namespace {

constexpr int kBins = 16;
constexpr int kMaxDepth = 56;      // stack use <= depth + 1 < 64
constexpr int kMaxLeaf = 8;        // leaf cap of the SAH termination
constexpr int kParallelMin = 1 << 15;

struct Aabb {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
  float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  void grow(const float* p) {
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
  }
  void grow(const Aabb& b) {
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], b.lo[a]); hi[a] = std::max(hi[a], b.hi[a]); }
  }
  float area() const {
    float d[3];
    for (int a = 0; a < 3; ++a) d[a] = std::max(0.f, hi[a] - lo[a]);
    return d[0] * d[1] + d[1] * d[2] + d[2] * d[0];
  }
};

struct TriRef {
  Aabb box;
  float c[3];
};

struct TreeNode {
  Aabb box;
  std::unique_ptr<TreeNode> kid[2];
  uint32_t first = 0, count = 0;
};

class Builder {
 public:
  Builder(std::vector<TriRef>& tris, std::vector<uint32_t>& order) : tris_(tris), order_(order) {}

  std::unique_ptr<TreeNode> build(uint32_t begin, uint32_t end, int depth) {
    auto node = std::make_unique<TreeNode>();
    Aabb cb;
    for (uint32_t i = begin; i < end; ++i) {
      node->box.grow(tris_[order_[i]].box);
      cb.grow(tris_[order_[i]].c);
    }
    uint32_t n = end - begin;
    node->first = begin;
    node->count = n;
    if (n <= 1 || depth >= kMaxDepth) return node;

    // binned SAH over the three centroid axes
    int best_axis = -1, best_split = -1;
    float best_cost = FLT_MAX;
    for (int a = 0; a < 3; ++a) {
      float ext = cb.hi[a] - cb.lo[a];
      if (!(ext > 0.f)) continue;
      Aabb bin_box[kBins];
      uint32_t bin_cnt[kBins] = {};
      float scale = kBins / ext;
      for (uint32_t i = begin; i < end; ++i) {
        const TriRef& t = tris_[order_[i]];
        int b = std::min(kBins - 1, int((t.c[a] - cb.lo[a]) * scale));
        bin_cnt[b]++;
        bin_box[b].grow(t.box);
      }
      float right_area[kBins];
      uint32_t right_cnt[kBins];
      Aabb acc;
      uint32_t cnt = 0;
      for (int b = kBins - 1; b > 0; --b) {
        acc.grow(bin_box[b]);
        cnt += bin_cnt[b];
        right_area[b] = acc.area();
        right_cnt[b] = cnt;
      }
      acc = Aabb();
      cnt = 0;
      for (int b = 0; b < kBins - 1; ++b) {
        acc.grow(bin_box[b]);
        cnt += bin_cnt[b];
        if (cnt == 0 || right_cnt[b + 1] == 0) continue;
        float cost = acc.area() * cnt + right_area[b + 1] * right_cnt[b + 1];
        if (cost < best_cost) { best_cost = cost; best_axis = a; best_split = b; }
      }
    }
    float leaf_cost = node->box.area() * n;
    if (best_axis < 0) {
      if (n <= uint32_t(kMaxLeaf)) return node;
      return split_median(std::move(node), begin, end, depth);  // coincident centroids
    }
    // SAH with unit traversal / intersection costs (relative to parent area)
    float split_cost = node->box.area() + best_cost;
    if (n <= uint32_t(kMaxLeaf) && leaf_cost <= split_cost) return node;

    float ext = cb.hi[best_axis] - cb.lo[best_axis];
    float scale = kBins / ext;
    auto mid_it = std::partition(order_.begin() + begin, order_.begin() + end, [&](uint32_t ti) {
      const TriRef& t = tris_[ti];
      int b = std::min(kBins - 1, int((t.c[best_axis] - cb.lo[best_axis]) * scale));
      return b <= best_split;
    });
    uint32_t mid = uint32_t(mid_it - order_.begin());
    if (mid == begin || mid == end) return split_median(std::move(node), begin, end, depth);
    return recurse(std::move(node), begin, mid, end, depth);
  }

 private:
  std::unique_ptr<TreeNode> split_median(std::unique_ptr<TreeNode> node, uint32_t begin, uint32_t end, int depth) {
    uint32_t mid = begin + (end - begin) / 2;
    return recurse(std::move(node), begin, mid, end, depth);
  }

  std::unique_ptr<TreeNode> recurse(std::unique_ptr<TreeNode> node, uint32_t begin, uint32_t mid, uint32_t end,
                                    int depth) {
    node->count = 0;
    bool parallel = false;
    if (end - begin >= uint32_t(kParallelMin)) {
      if (active_.fetch_add(1) < int(std::thread::hardware_concurrency())) parallel = true;
      else active_.fetch_sub(1);
    }
    if (parallel) {
      auto fut = std::async(std::launch::async, [&] { return build(begin, mid, depth + 1); });
      node->kid[1] = build(mid, end, depth + 1);
      node->kid[0] = fut.get();
      active_.fetch_sub(1);
    } else {
      node->kid[0] = build(begin, mid, depth + 1);
      node->kid[1] = build(mid, end, depth + 1);
    }
    return node;
  }

  std::vector<TriRef>& tris_;
  std::vector<uint32_t>& order_;
  std::atomic<int> active_{0};
};

void put_box(float* dst, const Aabb& b, float w_lo, float w_hi, int slot) {
  float* lo = dst + 4 * slot;
  float* hi = dst + 4 * (slot + 1);
  lo[0] = b.lo[0]; lo[1] = b.lo[1]; lo[2] = b.lo[2]; lo[3] = w_lo;
  hi[0] = b.hi[0]; hi[1] = b.hi[1]; hi[2] = b.hi[2]; hi[3] = w_hi;
}

}  // namespace

struct BvhResult {
  std::vector<float> nodes;     // 16 floats per node
  std::vector<int32_t> remap;   // one mesh triangle index per leaf slot
  uint32_t depth = 0;
  uint32_t triangles = 0;
  std::string error;
};

static uint32_t flatten(const TreeNode* n, std::vector<float>& out, uint32_t depth, uint32_t* max_depth) {
  uint32_t self = uint32_t(out.size() / 16);
  out.resize(out.size() + 16, 0.f);
  *max_depth = std::max(*max_depth, depth);
  if (!n->kid[0]) {
    float* d = &out[size_t(self) * 16];
    d[3] = 0.f; d[7] = 0.f;
    d[11] = float(n->count);
    d[15] = float(n->first);
    return self;
  }
  uint32_t l = flatten(n->kid[0].get(), out, depth + 1, max_depth);
  uint32_t r = flatten(n->kid[1].get(), out, depth + 1, max_depth);
  float* d = &out[size_t(self) * 16];
  put_box(d, n->kid[0]->box, float(l), float(r), 0);
  put_box(d, n->kid[1]->box, 0.f, 0.f, 2);
  d[11] = 0.f;  // cnt = 0 -> interior
  d[15] = 0.f;
  return self;
}

BvhResult* build_bvh(const float* positions, uint32_t num_vertices, uint32_t stride, const uint32_t* indices,
                     uint32_t num_indices) {
  auto* res = new BvhResult();
  if (!positions || stride < 3 || num_vertices == 0) { res->error = "empty or malformed position buffer"; return res; }
  if (!indices || num_indices == 0 || num_indices % 3) { res->error = "index buffer does not describe whole triangles"; return res; }
  uint32_t ntri = num_indices / 3;
  if (2ull * ntri > (1ull << 24)) { res->error = "scene exceeds 2^23 triangles (float-encoded node indices)"; return res; }
  std::vector<TriRef> tris(ntri);
  for (uint32_t t = 0; t < ntri; ++t) {
    TriRef& r = tris[t];
    for (int k = 0; k < 3; ++k) {
      uint32_t vi = indices[3 * t + k];
      if (vi >= num_vertices) { res->error = "index out of range at triangle " + std::to_string(t); return res; }
      r.box.grow(positions + size_t(vi) * stride);
    }
    for (int a = 0; a < 3; ++a) r.c[a] = 0.5f * (r.box.lo[a] + r.box.hi[a]);
  }
  std::vector<uint32_t> order(ntri);
  for (uint32_t i = 0; i < ntri; ++i) order[i] = i;
  Builder b(tris, order);
  std::unique_ptr<TreeNode> root = b.build(0, ntri, 0);
  res->nodes.reserve(size_t(2 * ntri) * 16);
  flatten(root.get(), res->nodes, 0, &res->depth);
  res->remap.assign(order.begin(), order.end());
  res->triangles = ntri;
  return res;
}

}  // namespace dspbr

// ---- C ABI (declared in include/dspbr.h) -----------------------------------
using dspbr::BvhResult;

extern "C" int dspbr_bvh_build(const float* positions, uint32_t num_vertices, uint32_t vertex_stride_floats,
                               const uint32_t* indices, uint32_t num_indices, dspbr_bvh** out) {
  if (!out) return DSPBR_ERR_INVALID;
  BvhResult* r = dspbr::build_bvh(positions, num_vertices, vertex_stride_floats, indices, num_indices);
  *out = reinterpret_cast<dspbr_bvh*>(r);
  return r->error.empty() ? DSPBR_OK : DSPBR_ERR_INVALID;
}

extern "C" int dspbr_bvh_info(const dspbr_bvh* h, uint32_t* num_nodes, uint32_t* num_indices, uint32_t* depth,
                              uint32_t* num_triangles) {
  auto* r = reinterpret_cast<const BvhResult*>(h);
  if (!r) return DSPBR_ERR_INVALID;
  if (num_nodes) *num_nodes = uint32_t(r->nodes.size() / 16);
  if (num_indices) *num_indices = uint32_t(r->remap.size());
  if (depth) *depth = r->depth;
  if (num_triangles) *num_triangles = r->triangles;
  return r->error.empty() ? DSPBR_OK : DSPBR_ERR_INVALID;
}

extern "C" int dspbr_bvh_copy(const dspbr_bvh* h, float* nodes, int32_t* indices) {
  auto* r = reinterpret_cast<const BvhResult*>(h);
  if (!r || !r->error.empty()) return DSPBR_ERR_INVALID;
  if (nodes) std::memcpy(nodes, r->nodes.data(), r->nodes.size() * sizeof(float));
  if (indices) std::memcpy(indices, r->remap.data(), r->remap.size() * sizeof(int32_t));
  return DSPBR_OK;
}

extern "C" int dspbr_bvh_error(const dspbr_bvh* h, char* buf, size_t size) {
  auto* r = reinterpret_cast<const BvhResult*>(h);
  if (!r || !buf || size == 0) return DSPBR_ERR_INVALID;
  std::snprintf(buf, size, "%s", r->error.c_str());
  return DSPBR_OK;
}

extern "C" void dspbr_bvh_free(dspbr_bvh* h) { delete reinterpret_cast<BvhResult*>(h); }
