// BVH construction and 4-wide collapse on the device (bvh_gpu.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "host.h"

namespace dspbr {

// A binary BVH in the device layout of DevScene::nodes (reference layout,
// child / count / first as int bits) and its leaf-slot remap.
struct DeviceBvh {
  DevBuf<float4> nodes;  // 4 float4 per node
  DevBuf<int32_t> remap;
  uint32_t num_nodes = 0, num_slots = 0;
};

// Linear BVH over the triangles (verts: 5 float4 per vertex, position in the
// first; indices: 3 per triangle).  Synchronises `st` before returning.
int build_bvh_device(const float4* verts, const uint32_t* indices, uint32_t ntris, cudaStream_t st, DeviceBvh* out,
                     Status& s);

// Binned-SAH BVH over the triangles with the host builder's rules
// (bvh_build.cpp), built level by level on the device; same inputs and output
// layout as build_bvh_device.  Synchronises `st` before returning.
int build_bvh_device_sah(const float4* verts, const uint32_t* indices, uint32_t ntris, cudaStream_t st,
                         DeviceBvh* out, Status& s);

// 4-wide collapse of a well-formed binary BVH already on the device (the same
// rule as collapse_bvh4, level by level).  wnodes: 8 float4 per wide node.
struct DeviceWideBvh {
  DevBuf<float4> nodes;
  DevBuf<int2> leaves;
  int32_t root = 0;
  uint32_t num_nodes = 0, num_leaves = 0;
};
int collapse_bvh4_device(const DeviceBvh& bin, cudaStream_t st, DeviceWideBvh* out, Status& s);

// Compressed 8-wide BVH (traversal: device.cuh cw8_step) built on the device
// from a binary BVH in the reference layout and its leaf-ordered triangle
// records.  Node: 5 x 16 B (per axis a frame P and power-of-two step, per
// child six plane bytes, the inner-child mask, the first inner child's index
// and the first leaf record's index, and per child its record count).  Leaf
// records: a header (the leaf's exact box and its slot count) and then the
// triangle records of the leaf's slots.  Leaves nothing in `out` (and returns
// DSPBR_OK) when the tree cannot be compressed: a leaf root, an axis no frame
// fits, a malformed tree.  Synchronises `st`.
struct DeviceCw8 {
  DevBuf<uint4> nodes;  // 5 per node
  DevBuf<float4> recs;  // 3 per record
  uint32_t num_nodes = 0, num_recs = 0, levels = 0;
};
int build_cw8_device(const float4* bin_nodes, uint32_t num_nodes, uint32_t num_slots, const float4* tris,
                     cudaStream_t st, DeviceCw8* out, Status& s);

// Refit after the vertices moved (indices unchanged): the boxes of the binary
// tree (reference layout) and of the 4-wide tree are recomputed bottom-up from
// their leaves' triangles, keeping both topologies, and the leaf-ordered
// triangle records are gathered again.  remap: the leaf-slot remap, or null to
// recover it from the records.  Synchronises `st`.
int refit_scene_device(float4* nodes, uint32_t num_nodes, uint32_t num_slots, float4* wnodes, uint32_t num_wide,
                       const int2* wleaves, float4* tris, const int32_t* remap, const float4* verts,
                       const uint32_t* indices, uint32_t ntris, cudaStream_t st, Status& s);

}  // namespace dspbr
