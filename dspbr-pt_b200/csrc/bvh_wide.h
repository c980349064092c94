// 4-wide BVH collapsed from the reference's binary BVH (bvh_wide.cpp).
#pragma once
#include <stdint.h>

#include <vector>

namespace dspbr {

constexpr int kWideMaxLeafTris = 64;  // MAX_TRIANGLES_PER_LEAF (bvh.glsl:10)

// One wide node = 128 bytes = 8 float4 on the device: the boxes of up to four
// children as structure of arrays, the children, and how many are used.
// child >= 0: wide node index; child < 0: leaf ~index into the leaf table.
struct alignas(16) WideNode4 {
  float lo_x[4], lo_y[4], lo_z[4];
  float hi_x[4], hi_y[4], hi_z[4];
  int32_t child[4];
  int32_t count;
  int32_t pad[3];
};
static_assert(sizeof(WideNode4) == 128, "wide node is one 128-byte line");

// Leaf-slot range [begin, end) of a binary leaf, already clipped as the
// reference's leaf loop clips it.
struct WideLeaf {
  int32_t begin, end;
};

struct WideBvh {
  std::vector<WideNode4> nodes;
  std::vector<WideLeaf> leaves;
  int32_t root = 0;  // >= 0: wide node; < 0: the binary root is a leaf (~leaf index)
};

WideBvh collapse_bvh4(const float* nodes, uint32_t num_nodes, uint32_t num_slots);

}  // namespace dspbr
