// BVH construction on the device, emitting the reference's binary node layout
// (bvh.glsl:1-6) so that every later stage -- the leaf triangle gather, the
// 4-wide collapse, both traversals -- is unchanged.  Two builders: the binned
// SAH with the host builder's rules (build_bvh_device_sah, below) and a
// linear BVH (build_bvh_device).
//
// The reference builds its BVH on the host with TinyBVH (tinybvh_builder.ts);
// the host binned-SAH builder here (bvh_build.cpp) plays that role.  The
// device binned SAH builds the same tree and is the default for scenes
// created without a BVH: for large scenes admitted while others render, a
// host build of seconds dominates the time to the first frame.  The linear
// BVH trades some tree quality for the fastest build:
//   1. per triangle: bounds and centroid; centroid bounds of the scene;
//   2. 63-bit Morton codes of the centroids (21 bits per axis), sorted with
//      the triangle index (CUB radix sort);
//   3. the radix tree over the sorted codes (Karras, "Maximizing parallelism
//      in the construction of BVHs, octrees, and k-d trees", HPG 2012), equal
//      codes ordered by position;
//   4. bounds and triangle counts bottom-up: each leaf walks towards the root,
//      the second child to arrive at a node computes its union;
//   5. output: subtrees of at most kLeafMax triangles become leaves (a
//      subtree is a contiguous range of the sorted triangles); the other
//      nodes store the boxes of their two children.
// Node ids: internal node i -> i, triangle leaf j -> (n - 1) + j, so the root
// is node 0 as the reference requires; nodes inside collapsed subtrees are
// unreachable and stay zero.
#include <cuda_runtime.h>

#include <algorithm>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "bvh_gpu.h"
#include "kernels.h"

namespace dspbr {

namespace {

constexpr int kLeafMax = 4;

__device__ __forceinline__ uint64_t spread21(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

struct Box {
  float lo[3], hi[3];
};

__global__ void k_tri_bounds(const float4* __restrict__ verts, const uint32_t* __restrict__ idx, uint32_t n,
                             float4* __restrict__ lo, float4* __restrict__ hi, float* __restrict__ block_bounds) {
  __shared__ float red[6][256];
  float c_lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, c_hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    float4 a = verts[5 * size_t(idx[3 * size_t(t)])], b = verts[5 * size_t(idx[3 * size_t(t) + 1])],
           c = verts[5 * size_t(idx[3 * size_t(t) + 2])];
    float4 l = make_float4(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)), 0.f);
    float4 h = make_float4(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)), 0.f);
    lo[t] = l;
    hi[t] = h;
    float cx = 0.5f * (l.x + h.x), cy = 0.5f * (l.y + h.y), cz = 0.5f * (l.z + h.z);
    c_lo[0] = fminf(c_lo[0], cx); c_lo[1] = fminf(c_lo[1], cy); c_lo[2] = fminf(c_lo[2], cz);
    c_hi[0] = fmaxf(c_hi[0], cx); c_hi[1] = fmaxf(c_hi[1], cy); c_hi[2] = fmaxf(c_hi[2], cz);
  }
  for (int k = 0; k < 3; ++k) {
    red[k][threadIdx.x] = c_lo[k];
    red[3 + k][threadIdx.x] = c_hi[k];
  }
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 3; ++k) {
        red[k][threadIdx.x] = fminf(red[k][threadIdx.x], red[k][threadIdx.x + s]);
        red[3 + k][threadIdx.x] = fmaxf(red[3 + k][threadIdx.x], red[3 + k][threadIdx.x + s]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) block_bounds[6 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_morton(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
                         const float* __restrict__ block_bounds, int nblocks, uint64_t* __restrict__ keys,
                         uint32_t* __restrict__ ids) {
  __shared__ float sb[6];
  if (threadIdx.x < 6) {
    float v = threadIdx.x < 3 ? 3.4e38f : -3.4e38f;
    for (int b = 0; b < nblocks; ++b) {
      float x = block_bounds[6 * b + threadIdx.x];
      v = threadIdx.x < 3 ? fminf(v, x) : fmaxf(v, x);
    }
    sb[threadIdx.x] = v;
  }
  __syncthreads();
  const float ex = fmaxf(sb[3] - sb[0], 1e-30f), ey = fmaxf(sb[4] - sb[1], 1e-30f), ez = fmaxf(sb[5] - sb[2], 1e-30f);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    float4 l = lo[t], h = hi[t];
    float cx = (0.5f * (l.x + h.x) - sb[0]) / ex, cy = (0.5f * (l.y + h.y) - sb[1]) / ey,
          cz = (0.5f * (l.z + h.z) - sb[2]) / ez;
    const float m = 2097151.f;  // 2^21 - 1
    uint32_t ix = uint32_t(fminf(fmaxf(cx * m, 0.f), m)), iy = uint32_t(fminf(fmaxf(cy * m, 0.f), m)),
             iz = uint32_t(fminf(fmaxf(cz * m, 0.f), m));
    keys[t] = spread21(ix) << 2 | spread21(iy) << 1 | spread21(iz);
    ids[t] = t;
  }
}

// common prefix length of keys i and j, extended by the index for equal keys
__device__ __forceinline__ int delta(const uint64_t* keys, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint64_t a = keys[i], b = keys[j];
  if (a == b) return 64 + __clz(uint32_t(i ^ j));
  return __clzll(a ^ b);
}

// Karras 2012: internal node i covers [first, last] of the sorted leaves and
// splits after `split`.  child >= 0: internal node; child < 0: leaf ~index.
__global__ void k_radix_tree(const uint64_t* __restrict__ keys, int n, int2* __restrict__ child,
                             int2* __restrict__ range, int* __restrict__ parent) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
    int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;  // bounded: lmax <= 2n
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
      if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s = 0;
    int len = l;
    for (int t = (len + 1) >> 1;; t = (t + 1) >> 1) {
      if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
      if (t == 1) break;
    }
    int split = i + s * d + min(d, 0);
    int first = min(i, j), last = max(i, j);
    int left = (first == split) ? ~split : split;
    int right = (last == split + 1) ? ~(split + 1) : split + 1;
    child[i] = make_int2(left, right);
    range[i] = make_int2(first, last);
    if (left >= 0) parent[left] = i;
    else parent[(n - 1) + ~left] = i;
    if (right >= 0) parent[right] = i;
    else parent[(n - 1) + ~right] = i;
  }
}

// Bounds and triangle counts bottom-up.  node_lo/hi/count index: internal i,
// leaf j at (n - 1) + j.  flags: one arrival counter per internal node.
__global__ void k_bounds_up(const float4* __restrict__ tlo, const float4* __restrict__ thi,
                            const uint32_t* __restrict__ ids, int n, const int2* __restrict__ child,
                            const int* __restrict__ parent, float4* node_lo, float4* node_hi, int* count,
                            int* flags) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int leaf = (n - 1) + j;
    node_lo[leaf] = tlo[ids[j]];
    node_hi[leaf] = thi[ids[j]];
    count[leaf] = 1;
    __threadfence();
    int p = parent[leaf];
    // at most depth <= n - 1 steps; the second arrival at a node continues
    for (int steps = 0; p >= 0 && steps < n; ++steps) {
      if (atomicAdd(&flags[p], 1) == 0) break;
      __threadfence();
      const int2 c = child[p];
      const int a = c.x >= 0 ? c.x : (n - 1) + ~c.x, b = c.y >= 0 ? c.y : (n - 1) + ~c.y;
      const float4 la = __ldcg(node_lo + a), ha = __ldcg(node_hi + a), lb = __ldcg(node_lo + b),
                   hb = __ldcg(node_hi + b);
      node_lo[p] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), 0.f);
      node_hi[p] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.f);
      count[p] = __ldcg(count + a) + __ldcg(count + b);
      __threadfence();
      p = p == 0 ? -1 : parent[p];
    }
  }
}

__device__ __forceinline__ float ibits(int v) { return __int_as_float(v); }

// Reference-layout nodes (int bits in lanes 3, 7, 11, 15) and the leaf-slot
// remap (sorted triangle ids).
__global__ void k_emit(int n, const int2* __restrict__ child, const int2* __restrict__ range,
                       const float4* __restrict__ node_lo, const float4* __restrict__ node_hi,
                       const int* __restrict__ count, const uint32_t* __restrict__ ids, float4* __restrict__ nodes,
                       int32_t* __restrict__ remap) {
  const int total = 2 * n - 1;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
    if (v < n) remap[v] = int32_t(ids[v]);
    float4* o = nodes + 4 * size_t(v);
    const bool is_leaf_prim = v >= n - 1;
    const int cnt = count[v];
    // a node is emitted as a leaf when its subtree is small (or it is a triangle)
    const bool as_leaf = is_leaf_prim || cnt <= kLeafMax;
    if (as_leaf) {
      const int first = is_leaf_prim ? v - (n - 1) : range[v].x;
      o[0] = make_float4(0.f, 0.f, 0.f, ibits(0));
      o[1] = make_float4(0.f, 0.f, 0.f, ibits(0));
      o[2] = make_float4(0.f, 0.f, 0.f, ibits(cnt));
      o[3] = make_float4(0.f, 0.f, 0.f, ibits(first));
      continue;
    }
    const int2 c = child[v];
    const int a = c.x >= 0 ? c.x : (n - 1) + ~c.x, b = c.y >= 0 ? c.y : (n - 1) + ~c.y;
    const float4 la = node_lo[a], ha = node_hi[a], lb = node_lo[b], hb = node_hi[b];
    o[0] = make_float4(la.x, la.y, la.z, ibits(a));
    o[1] = make_float4(ha.x, ha.y, ha.z, ibits(b));
    o[2] = make_float4(lb.x, lb.y, lb.z, ibits(0));
    o[3] = make_float4(hb.x, hb.y, hb.z, ibits(0));
  }
}

// ---- 4-wide collapse, one frontier level per launch ---------------------------------------
struct WideCounters {
  int nodes, leaves, next;  // wide nodes and leaves allocated, entries of the next frontier
};

__device__ __forceinline__ int bin_int(const float4* nodes, int n, int lane) {
  return __float_as_int(reinterpret_cast<const float*>(nodes + 4 * size_t(n))[lane]);
}

__device__ __forceinline__ float box_area(float lx, float ly, float lz, float hx, float hy, float hz) {
  float dx = hx - lx, dy = hy - ly, dz = hz - lz;
  if (!(dx >= 0.f) || !(dy >= 0.f) || !(dz >= 0.f)) return 0.f;
  return dx * dy + dy * dz + dz * dx;
}

struct WChild {
  int node;
  float lo[3], hi[3];
};

// children of binary inner node n, as bvh_push_child would push them
__device__ int bin_children(const float4* nodes, uint32_t num_nodes, int n, WChild* out) {
  const float4 n0 = nodes[4 * size_t(n)], n1 = nodes[4 * size_t(n) + 1], n2 = nodes[4 * size_t(n) + 2],
               n3 = nodes[4 * size_t(n) + 3];
  const int l = __float_as_int(n0.w), r = __float_as_int(n1.w);
  int m = 0;
  if (l >= 0 && uint32_t(l) < num_nodes && l != n) out[m++] = {l, {n0.x, n0.y, n0.z}, {n1.x, n1.y, n1.z}};
  if (r >= 0 && uint32_t(r) < num_nodes && r != n) out[m++] = {r, {n2.x, n2.y, n2.z}, {n3.x, n3.y, n3.z}};
  return m;
}

__global__ void k_collapse_level(const float4* __restrict__ bin, uint32_t num_nodes, uint32_t num_slots,
                                 const int2* __restrict__ frontier, int count, int2* __restrict__ next,
                                 float4* __restrict__ wnodes, int2* __restrict__ wleaves, WideCounters* ctr) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < count; f += gridDim.x * blockDim.x) {
    const int2 e = frontier[f];  // (binary inner node, wide slot)
    WChild kids[4];
    int nk = bin_children(bin, num_nodes, e.x, kids);
    for (int guard = 0; guard < 4; ++guard) {  // open the largest inner child while there is room
      int best = -1;
      float best_area = -1.f;
      WChild grand[2];
      for (int k = 0; k < nk; ++k) {
        if (bin_int(bin, kids[k].node, 11) > 0) continue;  // a leaf
        if (nk - 1 + bin_children(bin, num_nodes, kids[k].node, grand) > 4) continue;
        float a = box_area(kids[k].lo[0], kids[k].lo[1], kids[k].lo[2], kids[k].hi[0], kids[k].hi[1], kids[k].hi[2]);
        if (a > best_area) {
          best_area = a;
          best = k;
        }
      }
      if (best < 0) break;
      const int ng = bin_children(bin, num_nodes, kids[best].node, grand);
      for (int k = best; k + 1 < nk; ++k) kids[k] = kids[k + 1];
      --nk;
      for (int k = 0; k < ng; ++k) kids[nk++] = grand[k];
    }
    float lo[3][4], hi[3][4];
    int ch[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k)
      for (int a = 0; a < 3; ++a) lo[a][k] = hi[a][k] = 0.f;
    for (int k = 0; k < nk; ++k) {
      for (int a = 0; a < 3; ++a) {
        lo[a][k] = kids[k].lo[a];
        hi[a][k] = kids[k].hi[a];
      }
      const int c = kids[k].node;
      const int cnt = bin_int(bin, c, 11);
      if (cnt > 0) {  // a leaf: the slot range the reference's leaf loop tests
        const int first = bin_int(bin, c, 15);
        long long b0 = first > 0 ? first : 0;
        long long b1 = (long long)first + (cnt < 64 ? cnt : 64);
        if (b1 > (long long)num_slots) b1 = num_slots;
        if (b1 < b0) b1 = b0;
        const int li = atomicAdd(&ctr->leaves, 1);
        wleaves[li] = make_int2(int(b0), int(b1));
        ch[k] = ~li;
      } else {
        const int wi = atomicAdd(&ctr->nodes, 1);
        next[atomicAdd(&ctr->next, 1)] = make_int2(c, wi);
        ch[k] = wi;
      }
    }
    float4* o = wnodes + 8 * size_t(e.y);
    o[0] = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
    o[1] = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
    o[2] = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
    o[3] = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
    o[4] = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
    o[5] = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
    o[6] = make_float4(__int_as_float(ch[0]), __int_as_float(ch[1]), __int_as_float(ch[2]), __int_as_float(ch[3]));
    o[7] = make_float4(__int_as_float(nk), 0.f, 0.f, 0.f);
  }
}

// ---- compressed 8-wide BVH, one frontier level per launch ----------------------------------
constexpr int kLeafSlotsMax = 64;  // MAX_TRIANGLES_PER_LEAF (bvh.glsl:10)

struct Cw8Counters {
  int nodes, next, recs, error;  // nodes and leaf records allocated, next frontier entries, overflow
};

// the plane of byte q in a frame (P, 2^e): bit-identical to device.cuh cw8_plane
__device__ __forceinline__ float cw8_plane_q(uint32_t q, float scale, float p) {
  return fmaf(__uint_as_float(0x4B000000u | q), scale, p);
}

// The frame of one axis of a node box [lo, hi]: the smallest power-of-two
// step (up to 2^100) whose 256 planes reach from at most lo to at least hi.
__device__ bool cw8_frame(float lo, float hi, uint32_t& ebyte, float& p_out) {
  int e0;
  if (hi > lo) {
    e0 = int(floor(log2(double(hi) - double(lo)) - log2(255.0))) - 1;
  } else {
    int ex;
    frexpf(fabsf(lo) > 0.f ? lo : 1.f, &ex);
    e0 = ex - 40;
  }
  if (e0 < -100) e0 = -100;
  for (int e = e0; e <= 100; ++e) {
    const float scale = ldexpf(1.f, e);
    float p = __fsub_rn(lo, ldexpf(1.f, e + 23));
    for (int g = 0; g < 64 && cw8_plane_q(0u, scale, p) > lo; ++g) p = nextafterf(p, -INFINITY);
    if (cw8_plane_q(0u, scale, p) <= lo && cw8_plane_q(255u, scale, p) >= hi) {
      ebyte = uint32_t(e + 127);
      p_out = p;
      return true;
    }
  }
  return false;
}
// the largest byte whose plane is <= c, and the smallest whose plane is >= c
__device__ uint32_t cw8_qlo(float c, float scale, float p, float lo) {
  const double d = floor((double(c) - double(lo)) / double(scale));
  int q = int(fmin(255.0, fmax(0.0, d)));
  for (int g = 0; g < 256 && q > 0 && cw8_plane_q(q, scale, p) > c; ++g) --q;
  for (int g = 0; g < 256 && q < 255 && cw8_plane_q(q + 1, scale, p) <= c; ++g) ++q;
  return uint32_t(q);
}
__device__ uint32_t cw8_qhi(float c, float scale, float p, float lo) {
  const double d = ceil((double(c) - double(lo)) / double(scale));
  int q = int(fmin(255.0, fmax(0.0, d)));
  for (int g = 0; g < 256 && q < 255 && cw8_plane_q(q, scale, p) < c; ++g) ++q;
  for (int g = 0; g < 256 && q > 0 && cw8_plane_q(q - 1, scale, p) >= c; ++g) --q;
  return uint32_t(q);
}
__device__ __forceinline__ void cw8_setb(uint32_t* w, int k, uint32_t v) {
  w[k >> 2] = (w[k >> 2] & ~(0xFFu << (8 * (k & 3)))) | (v << (8 * (k & 3)));
}
// the leaf-slot range a binary leaf tests (the reference's leaf loop)
__device__ __forceinline__ void leaf_range(const float4* bin, uint32_t num_slots, int c, long long& b0, long long& b1) {
  const int cnt = bin_int(bin, c, 11), first = bin_int(bin, c, 15);
  b0 = first > 0 ? first : 0;
  b1 = (long long)first + (cnt < kLeafSlotsMax ? cnt : kLeafSlotsMax);
  if (b1 > (long long)num_slots) b1 = num_slots;
  if (b1 < b0) b1 = b0;
}

// records a binary leaf needs: a header and its slots
__global__ void k_cw8_count(const float4* __restrict__ bin, uint32_t num_nodes, uint32_t num_slots,
                            unsigned long long* total) {
  unsigned long long mine = 0;
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < num_nodes; n += gridDim.x * blockDim.x) {
    if (bin_int(bin, int(n), 11) <= 0) continue;
    long long b0, b1;
    leaf_range(bin, num_slots, int(n), b0, b1);
    mine += (unsigned long long)(b1 - b0) + 1ull;
  }
  if (mine) atomicAdd(total, mine);
}

// One level: each frontier entry (binary inner node, compressed node index)
// takes up to 8 children by opening its largest inner child while there is
// room (the 4-wide collapse's rule), places them in slots by the alignment of
// their centre with the slot's corner, quantises their boxes and allocates
// its inner children (contiguous node indices) and its leaf records.
__global__ void k_cw8_level(const float4* __restrict__ bin, uint32_t num_nodes, uint32_t num_slots,
                            const int2* __restrict__ frontier, int count, int2* __restrict__ next, int next_cap,
                            uint4* __restrict__ cnodes, int node_cap, float4* __restrict__ recs,
                            int32_t* __restrict__ rec_src, int rec_cap, Cw8Counters* ctr) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < count; f += gridDim.x * blockDim.x) {
    const int2 fe = frontier[f];
    WChild kids[8];
    int nk = bin_children(bin, num_nodes, fe.x, kids);
    for (int guard = 0; guard < 8; ++guard) {
      int best = -1;
      float best_area = -1.f;
      WChild grand[2];
      for (int k = 0; k < nk; ++k) {
        if (bin_int(bin, kids[k].node, 11) > 0) continue;
        if (nk - 1 + bin_children(bin, num_nodes, kids[k].node, grand) > 8) continue;
        const float a = box_area(kids[k].lo[0], kids[k].lo[1], kids[k].lo[2], kids[k].hi[0], kids[k].hi[1], kids[k].hi[2]);
        if (a > best_area) {
          best_area = a;
          best = k;
        }
      }
      if (best < 0) break;
      const int ng = bin_children(bin, num_nodes, kids[best].node, grand);
      for (int k = best; k + 1 < nk; ++k) kids[k] = kids[k + 1];
      --nk;
      for (int k = 0; k < ng; ++k) kids[nk++] = grand[k];
    }
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < nk; ++k)
      for (int a = 0; a < 3; ++a) {
        const float l = fminf(kids[k].lo[a], kids[k].hi[a]), h = fmaxf(kids[k].lo[a], kids[k].hi[a]);
        kids[k].lo[a] = l;
        kids[k].hi[a] = h;
        lo[a] = fminf(lo[a], l);
        hi[a] = fmaxf(hi[a], h);
      }
    int kid_in[8];
    bool used[8];
    for (int s = 0; s < 8; ++s) {
      kid_in[s] = -1;
      used[s] = false;
    }
    float pc[3];
    for (int a = 0; a < 3; ++a) pc[a] = 0.5f * lo[a] + 0.5f * hi[a];
    for (int r = 0; r < nk; ++r) {
      float bs = -INFINITY;
      int bk = -1, bsl = -1;
      for (int k = 0; k < nk; ++k) {
        if (used[k]) continue;
        for (int s = 0; s < 8; ++s) {
          if (kid_in[s] >= 0) continue;
          float sc = 0.f;
          for (int a = 0; a < 3; ++a) {
            const float c = 0.5f * kids[k].lo[a] + 0.5f * kids[k].hi[a] - pc[a];
            sc += ((s >> a) & 1) ? c : -c;
          }
          if (bk < 0 || sc > bs) {
            bs = sc;
            bk = k;
            bsl = s;
          }
        }
      }
      used[bk] = true;
      kid_in[bsl] = bk;
    }
    uint32_t eb[3];
    float P[3], S[3];
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      if (!cw8_frame(lo[a], hi[a], eb[a], P[a])) ok = false;
      S[a] = ok ? ldexpf(1.f, int(eb[a]) - 127) : 1.f;
    }
    if (!ok) {
      atomicOr(&ctr->error, 1);
      continue;
    }
    uint32_t imask = 0, meta[2] = {0u, 0u}, ql[3][2], qh[3][2];
    for (int a = 0; a < 3; ++a) {
      ql[a][0] = ql[a][1] = 0xFFFFFFFFu;  // empty slot: an inverted box on every axis
      qh[a][0] = qh[a][1] = 0u;
    }
    int ninner = 0, nrec = 0;
    for (int s = 0; s < 8; ++s) {
      const int k = kid_in[s];
      if (k < 0) continue;
      for (int a = 0; a < 3; ++a) {
        cw8_setb(ql[a], s, cw8_qlo(kids[k].lo[a], S[a], P[a], lo[a]));
        cw8_setb(qh[a], s, cw8_qhi(kids[k].hi[a], S[a], P[a], lo[a]));
      }
      if (bin_int(bin, kids[k].node, 11) > 0) {
        long long b0, b1;
        leaf_range(bin, num_slots, kids[k].node, b0, b1);
        cw8_setb(meta, s, uint32_t(b1 - b0) + 1u);
        nrec += int(b1 - b0) + 1;
      } else {
        imask |= 1u << s;
        ++ninner;
      }
    }
    const int cbase = ninner ? atomicAdd(&ctr->nodes, ninner) : 0;
    const int rbase = nrec ? atomicAdd(&ctr->recs, nrec) : 0;
    if (cbase + ninner > node_cap || rbase + nrec > rec_cap) {
      atomicOr(&ctr->error, 2);
      continue;
    }
    for (int s = 0, r = 0, at = rbase; s < 8; ++s) {
      const int k = kid_in[s];
      if (k < 0) continue;
      const int c = kids[k].node;
      if (bin_int(bin, c, 11) > 0) {
        long long b0, b1;
        leaf_range(bin, num_slots, c, b0, b1);
        const int n = int(b1 - b0);
        recs[3 * size_t(at)] = make_float4(kids[k].lo[0], kids[k].lo[1], kids[k].lo[2], __int_as_float(-1));
        recs[3 * size_t(at) + 1] = make_float4(kids[k].hi[0], kids[k].hi[1], kids[k].hi[2], __int_as_float(n));
        recs[3 * size_t(at) + 2] = make_float4(0.f, 0.f, 0.f, 0.f);
        rec_src[at] = -1;
        for (int j = 0; j < n; ++j) rec_src[at + 1 + j] = int(b0) + j;
        at += n + 1;
      } else {
        const int slot = atomicAdd(&ctr->next, 1);
        if (slot < next_cap) next[slot] = make_int2(c, cbase + r);
        else atomicOr(&ctr->error, 4);
        ++r;
      }
    }
    uint4* o = cnodes + 5 * size_t(fe.y);
    o[0] = make_uint4(__float_as_uint(P[0]), __float_as_uint(P[1]), __float_as_uint(P[2]),
                      eb[0] | eb[1] << 8 | eb[2] << 16 | imask << 24);
    o[1] = make_uint4(uint32_t(cbase), uint32_t(rbase), meta[0], meta[1]);
    o[2] = make_uint4(ql[0][0], ql[0][1], ql[1][0], ql[1][1]);
    o[3] = make_uint4(ql[2][0], ql[2][1], qh[0][0], qh[0][1]);
    o[4] = make_uint4(qh[1][0], qh[1][1], qh[2][0], qh[2][1]);
  }
}

// the triangle records of the leaves, in the compressed tree's order
__global__ void k_cw8_gather(const int32_t* __restrict__ rec_src, int n, const float4* __restrict__ tris,
                             float4* __restrict__ recs) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int src = rec_src[i];
    if (src < 0) continue;
    recs[3 * size_t(i)] = tris[3 * size_t(src)];
    recs[3 * size_t(i) + 1] = tris[3 * size_t(src) + 1];
    recs[3 * size_t(i) + 2] = tris[3 * size_t(src) + 2];
  }
}

// ---- refit: the same trees over moved vertices --------------------------------------------
constexpr int kMaxLeaf = 64;  // MAX_TRIANGLES_PER_LEAF (bvh.glsl:10): the slots a leaf test visits

// A box over the triangles of leaf slots [b0, b1); ids from the leaf-ordered
// triangle records (w = mesh triangle id bits, -1: a slot the traversal skips).
__device__ bool slot_box(const float4* __restrict__ tris, int b0, int b1, const float4* __restrict__ verts,
                         const uint32_t* __restrict__ idx, uint32_t ntris, float4& lo, float4& hi) {
  bool any = false;
  lo = make_float4(0.f, 0.f, 0.f, 0.f);
  hi = lo;
  for (int i = b0; i < b1; ++i) {
    const int id = __float_as_int(tris[3 * size_t(i)].w);
    if (id < 0 || uint32_t(id) >= ntris) continue;
    for (int k = 0; k < 3; ++k) {
      const float4 p = verts[5 * size_t(idx[3 * size_t(id) + k])];
      if (!any) {
        lo = make_float4(p.x, p.y, p.z, 0.f);
        hi = lo;
        any = true;
      } else {
        lo = make_float4(fminf(lo.x, p.x), fminf(lo.y, p.y), fminf(lo.z, p.z), 0.f);
        hi = make_float4(fmaxf(hi.x, p.x), fmaxf(hi.y, p.y), fmaxf(hi.z, p.z), 0.f);
      }
    }
  }
  return any;
}

__device__ __forceinline__ void box_union(float4& lo, float4& hi, bool& any, float4 l, float4 h) {
  if (!any) {
    lo = l;
    hi = h;
    any = true;
  } else {
    lo = make_float4(fminf(lo.x, l.x), fminf(lo.y, l.y), fminf(lo.z, l.z), 0.f);
    hi = make_float4(fmaxf(hi.x, h.x), fmaxf(hi.y, h.y), fmaxf(hi.z, h.z), 0.f);
  }
}

// Binary tree (reference layout: an inner node stores its children's boxes):
// parent links of valid children (child in range, not the node itself).
__global__ void k_refit_bin_parents(const float4* __restrict__ nodes, uint32_t nn, int* __restrict__ parent) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    const float4* o = nodes + 4 * size_t(i);
    if (__float_as_int(o[2].w) > 0) continue;  // leaf
    const int l = __float_as_int(o[0].w), r = __float_as_int(o[1].w);
    if (l >= 0 && uint32_t(l) < nn && uint32_t(l) != i) parent[l] = int(i);
    if (r >= 0 && uint32_t(r) < nn && uint32_t(r) != i) parent[r] = int(i);
  }
}

// Leaf boxes from their triangles (the slots the reference's leaf loop
// visits), then unions towards the root: the second child to arrive at an
// inner node writes both children's boxes into it.  A child without any
// triangle keeps the box its parent had.  Each walk is bounded by nn steps.
__global__ void k_refit_bin_up(float4* nodes, uint32_t nn, uint32_t nslots, const float4* __restrict__ tris,
                               const float4* __restrict__ verts, const uint32_t* __restrict__ idx, uint32_t ntris,
                               const int* __restrict__ parent, float4* box_lo, float4* box_hi, int* has_box,
                               int* flags) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    const float4* o = nodes + 4 * size_t(i);
    const int cnt = __float_as_int(o[2].w);
    if (cnt <= 0) continue;
    const int first = __float_as_int(o[3].w);
    const int b0 = max(first, 0);
    const long long end = (long long)first + (long long)min(cnt, kMaxLeaf);
    const int b1 = int(end < (long long)nslots ? end : (long long)nslots);
    float4 lo, hi;
    const bool any = slot_box(tris, b0, b1, verts, idx, ntris, lo, hi);
    box_lo[i] = lo;
    box_hi[i] = hi;
    has_box[i] = any ? 1 : 0;
    __threadfence();
    int p = parent[i];
    for (uint32_t steps = 0; p >= 0 && steps < nn; ++steps) {
      if (atomicAdd(&flags[p], 1) == 0) break;  // the sibling finishes this node
      __threadfence();
      float4* q = nodes + 4 * size_t(p);
      const int a = __float_as_int(q[0].w), c = __float_as_int(q[1].w);
      bool anyp = false;
      float4 plo = make_float4(0.f, 0.f, 0.f, 0.f), phi = plo;
      if (__ldcg(has_box + a)) {
        const float4 l = __ldcg(box_lo + a), h = __ldcg(box_hi + a);
        q[0] = make_float4(l.x, l.y, l.z, q[0].w);
        q[1] = make_float4(h.x, h.y, h.z, q[1].w);
        box_union(plo, phi, anyp, l, h);
      }
      if (__ldcg(has_box + c)) {
        const float4 l = __ldcg(box_lo + c), h = __ldcg(box_hi + c);
        q[2] = make_float4(l.x, l.y, l.z, q[2].w);
        q[3] = make_float4(h.x, h.y, h.z, q[3].w);
        box_union(plo, phi, anyp, l, h);
      }
      box_lo[p] = plo;
      box_hi[p] = phi;
      has_box[p] = anyp ? 1 : 0;
      __threadfence();
      p = parent[p];
    }
  }
}

// 4-wide tree: parent (node, child slot) of each wide node and the number of
// wide-node children of each node.
__global__ void k_refit_wide_parents(const float4* __restrict__ wnodes, uint32_t nw, int2* __restrict__ parent,
                                     int* __restrict__ inner) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += gridDim.x * blockDim.x) {
    const float4* o = wnodes + 8 * size_t(i);
    const int4 ch = *reinterpret_cast<const int4*>(o + 6);
    const int n = min(max(__float_as_int(o[7].x), 0), 4);
    const int c[4] = {ch.x, ch.y, ch.z, ch.w};
    int k_inner = 0;
    for (int k = 0; k < n; ++k)
      if (c[k] >= 0 && uint32_t(c[k]) < nw && uint32_t(c[k]) != i) {
        parent[c[k]] = make_int2(int(i), k);
        ++k_inner;
      }
    inner[i] = k_inner;
  }
}

__device__ __forceinline__ void wide_set_box(float4* o, int k, float4 lo, float4 hi) {
  float* f = reinterpret_cast<float*>(o);
  f[0 * 4 + k] = lo.x; f[1 * 4 + k] = lo.y; f[2 * 4 + k] = lo.z;
  f[3 * 4 + k] = hi.x; f[4 * 4 + k] = hi.y; f[5 * 4 + k] = hi.z;
}

// A wide node whose children are all leaves starts a walk: its leaf boxes,
// its own box into its parent's slot; the last wide-node child to arrive at a
// node finishes it (its leaf children, then its own box) and goes on.
__global__ void k_refit_wide_up(float4* wnodes, uint32_t nw, const int2* __restrict__ wleaves,
                                const float4* __restrict__ tris, const float4* __restrict__ verts,
                                const uint32_t* __restrict__ idx, uint32_t ntris, const int2* __restrict__ parent,
                                const int* __restrict__ inner, int* flags) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += gridDim.x * blockDim.x) {
    if (inner[i] != 0) continue;
    int v = int(i);
    for (uint32_t steps = 0; steps <= nw; ++steps) {
      float4* o = wnodes + 8 * size_t(v);
      const int4 ch = *reinterpret_cast<const int4*>(o + 6);
      const int n = min(max(__float_as_int(o[7].x), 0), 4);
      const int c[4] = {ch.x, ch.y, ch.z, ch.w};
      bool any = false;
      float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
      for (int k = 0; k < n; ++k) {
        float4 l, h;
        if (c[k] < 0) {  // leaf child: its triangles
          const int2 r = wleaves[~c[k]];
          if (!slot_box(tris, r.x, r.y, verts, idx, ntris, l, h)) continue;
          wide_set_box(o, k, l, h);
        } else {  // wide child: the box its walk left in this slot
          const float* f = reinterpret_cast<const float*>(o);
          l = make_float4(__ldcg(f + 0 * 4 + k), __ldcg(f + 1 * 4 + k), __ldcg(f + 2 * 4 + k), 0.f);
          h = make_float4(__ldcg(f + 3 * 4 + k), __ldcg(f + 4 * 4 + k), __ldcg(f + 5 * 4 + k), 0.f);
        }
        box_union(lo, hi, any, l, h);
      }
      const int2 pk = parent[v];
      if (pk.x < 0) break;  // the root
      if (any) wide_set_box(wnodes + 8 * size_t(pk.x), pk.y, lo, hi);
      __threadfence();
      if (atomicAdd(&flags[pk.x], 1) + 1 != inner[pk.x]) break;  // other children still to come
      __threadfence();
      v = pk.x;
    }
  }
}

// leaf-slot remap recovered from the leaf-ordered triangle records
__global__ void k_remap_from_tris(const float4* __restrict__ tris, uint32_t nslots, int32_t* __restrict__ remap) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nslots; i += gridDim.x * blockDim.x)
    remap[i] = __float_as_int(tris[3 * size_t(i)].w);
}

int grid(size_t n, int threads, int cap) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return int(b < size_t(cap) ? b : size_t(cap));
}

}  // namespace

int refit_scene_device(float4* nodes, uint32_t num_nodes, uint32_t num_slots, float4* wnodes, uint32_t num_wide,
                       const int2* wleaves, float4* tris, const int32_t* remap, const float4* verts,
                       const uint32_t* indices, uint32_t ntris, cudaStream_t st, Status& s) {
  DevBuf<int> parent, flags, has_box, inner;
  DevBuf<float4> lo, hi;
  DevBuf<int2> wparent;
  DevBuf<int32_t> own_remap;
  TRY_CUDA(s, parent.alloc(std::max<uint32_t>(num_nodes, 1)), "refit");
  TRY_CUDA(s, flags.alloc(std::max<uint32_t>(std::max(num_nodes, num_wide), 1)), "refit");
  TRY_CUDA(s, has_box.alloc(std::max<uint32_t>(num_nodes, 1)), "refit");
  TRY_CUDA(s, lo.alloc(std::max<uint32_t>(num_nodes, 1)), "refit");
  TRY_CUDA(s, hi.alloc(std::max<uint32_t>(num_nodes, 1)), "refit");
  // binary tree
  TRY_CUDA(s, cudaMemsetAsync(parent.p, 0xff, parent.bytes(), st), "refit");
  TRY_CUDA(s, cudaMemsetAsync(flags.p, 0, flags.bytes(), st), "refit");
  k_refit_bin_parents<<<grid(num_nodes, 256, 148 * 8), 256, 0, st>>>(nodes, num_nodes, parent.p);
  k_refit_bin_up<<<grid(num_nodes, 256, 148 * 8), 256, 0, st>>>(nodes, num_nodes, num_slots, tris, verts, indices,
                                                                ntris, parent.p, lo.p, hi.p, has_box.p, flags.p);
  TRY_CUDA(s, cudaGetLastError(), "refit");
  // 4-wide tree
  if (num_wide) {
    TRY_CUDA(s, wparent.alloc(num_wide), "refit");
    TRY_CUDA(s, inner.alloc(num_wide), "refit");
    TRY_CUDA(s, cudaMemsetAsync(wparent.p, 0xff, wparent.bytes(), st), "refit");
    TRY_CUDA(s, cudaMemsetAsync(flags.p, 0, flags.bytes(), st), "refit");
    k_refit_wide_parents<<<grid(num_wide, 256, 148 * 8), 256, 0, st>>>(wnodes, num_wide, wparent.p, inner.p);
    k_refit_wide_up<<<grid(num_wide, 256, 148 * 8), 256, 0, st>>>(wnodes, num_wide, wleaves, tris, verts, indices,
                                                                  ntris, wparent.p, inner.p, flags.p);
    TRY_CUDA(s, cudaGetLastError(), "refit");
  }
  // the leaf-ordered triangle records over the new positions
  if (!remap) {
    TRY_CUDA(s, own_remap.alloc(std::max<uint32_t>(num_slots, 1)), "refit");
    k_remap_from_tris<<<grid(num_slots, 256, 148 * 8), 256, 0, st>>>(tris, num_slots, own_remap.p);
    remap = own_remap.p;
  }
  if (num_slots) launch_gather_tris(verts, indices, remap, num_slots, ntris, tris, st);
  TRY_CUDA(s, cudaGetLastError(), "refit");
  TRY_CUDA(s, cudaStreamSynchronize(st), "refit");
  return DSPBR_OK;
}

int build_bvh_device(const float4* verts, const uint32_t* indices, uint32_t ntris, cudaStream_t st, DeviceBvh* out,
                     Status& s) {
  if (ntris == 0) return s.fail(DSPBR_ERR_INVALID, "device BVH: no triangles");
  if (ntris > (1u << 28)) return s.fail(DSPBR_ERR_INVALID, "device BVH: too many triangles");
  const int n = int(ntris);
  const int total = 2 * n - 1;
  DevBuf<float4> tlo, thi, nlo, nhi;
  DevBuf<float> bb;
  DevBuf<uint64_t> keys, keys2;
  DevBuf<uint32_t> ids, ids2;
  DevBuf<int2> child, range;
  DevBuf<int> parent, count, flags;
  const int nb = grid(ntris, 256, 148 * 4);
  TRY_CUDA(s, tlo.alloc(n), "device BVH");
  TRY_CUDA(s, thi.alloc(n), "device BVH");
  TRY_CUDA(s, bb.alloc(6 * size_t(nb)), "device BVH");
  TRY_CUDA(s, keys.alloc(n), "device BVH");
  TRY_CUDA(s, keys2.alloc(n), "device BVH");
  TRY_CUDA(s, ids.alloc(n), "device BVH");
  TRY_CUDA(s, ids2.alloc(n), "device BVH");
  TRY_CUDA(s, nlo.alloc(total), "device BVH");
  TRY_CUDA(s, nhi.alloc(total), "device BVH");
  TRY_CUDA(s, count.alloc(total), "device BVH");
  TRY_CUDA(s, parent.alloc(total), "device BVH");
  TRY_CUDA(s, child.alloc(std::max(n - 1, 1)), "device BVH");
  TRY_CUDA(s, range.alloc(std::max(n - 1, 1)), "device BVH");
  TRY_CUDA(s, flags.alloc(std::max(n - 1, 1)), "device BVH");
  TRY_CUDA(s, out->nodes.alloc(size_t(total) * 4), "device BVH");
  TRY_CUDA(s, out->remap.alloc(n), "device BVH");
  k_tri_bounds<<<nb, 256, 0, st>>>(verts, indices, ntris, tlo.p, thi.p, bb.p);
  k_morton<<<grid(ntris, 256, 148 * 8), 256, 0, st>>>(tlo.p, thi.p, ntris, bb.p, nb, keys.p, ids.p);
  size_t temp = 0;
  TRY_CUDA(s, cub::DeviceRadixSort::SortPairs(nullptr, temp, keys.p, keys2.p, ids.p, ids2.p, n, 0, 63, st),
           "device BVH sort");
  DevBuf<unsigned char> tmp;
  TRY_CUDA(s, tmp.alloc(std::max<size_t>(temp, 1)), "device BVH");
  TRY_CUDA(s, cub::DeviceRadixSort::SortPairs(tmp.p, temp, keys.p, keys2.p, ids.p, ids2.p, n, 0, 63, st),
           "device BVH sort");
  TRY_CUDA(s, cudaMemsetAsync(parent.p, 0xff, parent.bytes(), st), "device BVH");
  TRY_CUDA(s, cudaMemsetAsync(flags.p, 0, flags.bytes(), st), "device BVH");
  if (n > 1) k_radix_tree<<<grid(n - 1, 256, 148 * 8), 256, 0, st>>>(keys2.p, n, child.p, range.p, parent.p);
  k_bounds_up<<<grid(n, 256, 148 * 8), 256, 0, st>>>(tlo.p, thi.p, ids2.p, n, child.p, parent.p, nlo.p, nhi.p,
                                                      count.p, flags.p);
  TRY_CUDA(s, cudaMemsetAsync(out->nodes.p, 0, out->nodes.bytes(), st), "device BVH");
  k_emit<<<grid(total, 256, 148 * 8), 256, 0, st>>>(n, child.p, range.p, nlo.p, nhi.p, count.p, ids2.p, out->nodes.p,
                                                    out->remap.p);
  TRY_CUDA(s, cudaGetLastError(), "device BVH");
  // the temporaries are freed at return: wait for the kernels that use them
  TRY_CUDA(s, cudaStreamSynchronize(st), "device BVH");
  out->num_nodes = uint32_t(total);
  out->num_slots = uint32_t(n);
  return DSPBR_OK;
}

// ---- binned SAH on the device, level by level ----------------------------------------------
// The host builder's rules (bvh_build.cpp: 16 bins per centroid axis, SAH
// with unit costs relative to the parent's area, a leaf when the SAH prefers
// it at <= 8 triangles, a median split when the centroids coincide, depth
// <= 56), evaluated for every open node of a level at once:
//   1. binning: each triangle of an open node adds itself to its node's bins
//      (count, box, centroid box per axis and bin) with integer atomics on
//      order-preserving encodings of the floats (min / max are exact and
//      independent of the order);
//   2. one thread per open node evaluates the 3 x 15 candidate planes and
//      decides leaf / split / median split;
//   3. child ids: an exclusive scan over the level (2 per split node), so
//      the ids and the tree do not depend on scheduling; the children of the
//      k-th split node are consecutive and ordered like the parent ranges;
//   4. a stable partition of every split node's range (an exclusive scan of
//      goes-left flags over all slots) into the left and right child ranges.
// Node records are written in the reference layout as nodes are decided.
constexpr int kSahBins = 16;
constexpr int kSahMaxLeaf = 8;
constexpr int kSahMaxDepth = 56;
constexpr int kBinWords = 13;  // count, box lo / hi, centroid lo / hi (encoded)

__device__ __forceinline__ int f2o(float f) {  // order-preserving float -> int
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

struct SahNode {
  float4 lo, hi;    // box
  float4 clo, chi;  // centroid box
  int begin, end;   // slot range
  int depth, pad;
};

// the bin of centroid c along one axis of the centroid box [lo, lo + ext]
__device__ __forceinline__ int sah_bin(float c, float lo, float ext) {
  const int b = int((c - lo) * (float(kSahBins) / ext));
  return min(kSahBins - 1, max(0, b));
}

__device__ __forceinline__ float comp(const float4& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// Area and costs with every product and sum rounded on its own (no FMA
// contraction), as the host builder computes them: equal costs, equal planes.
__device__ __forceinline__ float sah_area(float lx, float ly, float lz, float hx, float hy, float hz) {
  const float dx = fmaxf(0.f, hx - lx), dy = fmaxf(0.f, hy - ly), dz = fmaxf(0.f, hz - lz);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}

__global__ void k_sah_init(uint32_t n, int* __restrict__ bins, uint32_t nbins_words) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nbins_words; i += gridDim.x * blockDim.x) {
    const uint32_t w = i % kBinWords;
    bins[i] = w == 0 ? 0 : ((w - 1) % 6 < 3 ? 0x7fffffff : int(0x80000000));
  }
}

// 1. binning of the triangles whose node is in the chunk [c_begin, c_end) of this level
__global__ void k_sah_bin(uint32_t n, const uint32_t* __restrict__ order, const int* __restrict__ pnode,
                          const float4* __restrict__ tlo, const float4* __restrict__ thi,
                          const SahNode* __restrict__ nodes, int c_begin, int c_end, int* __restrict__ bins) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int v = pnode[s];
    if (v < c_begin || v >= c_end) continue;
    const SahNode nd = nodes[v];
    const uint32_t t = order[s];
    const float4 l = tlo[t], h = thi[t];
    const float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
    int* nb = bins + size_t(v - c_begin) * (3 * kSahBins * kBinWords);
    for (int a = 0; a < 3; ++a) {
      const float lo = comp(nd.clo, a), ext = comp(nd.chi, a) - lo;
      if (!(ext > 0.f)) continue;
      int* w = nb + (a * kSahBins + sah_bin(c[a], lo, ext)) * kBinWords;
      atomicAdd(w, 1);
      atomicMin(w + 1, f2o(l.x)); atomicMin(w + 2, f2o(l.y)); atomicMin(w + 3, f2o(l.z));
      atomicMax(w + 4, f2o(h.x)); atomicMax(w + 5, f2o(h.y)); atomicMax(w + 6, f2o(h.z));
      atomicMin(w + 7, f2o(c[0])); atomicMin(w + 8, f2o(c[1])); atomicMin(w + 9, f2o(c[2]));
      atomicMax(w + 10, f2o(c[0])); atomicMax(w + 11, f2o(c[1])); atomicMax(w + 12, f2o(c[2]));
    }
  }
}

// 1'. the same for the first levels (few nodes, every triangle of the
// level in their bins): each block bins into shared memory, then adds its
// non-empty bins to the global ones, so that the global atomics per bin are
// one per block instead of one per triangle.
constexpr int kSharedBinNodes = 32;  // 32 nodes x 2.5 KB of bins
__global__ void k_sah_bin_shared(uint32_t n, const uint32_t* __restrict__ order, const int* __restrict__ pnode,
                                 const float4* __restrict__ tlo, const float4* __restrict__ thi,
                                 const SahNode* __restrict__ nodes, int c_begin, int c_end, int* __restrict__ bins) {
  extern __shared__ int sb[];
  const int nbins = (c_end - c_begin) * 3 * kSahBins;
  for (int i = threadIdx.x; i < nbins * kBinWords; i += blockDim.x) {
    const int w = i % kBinWords;
    sb[i] = w == 0 ? 0 : ((w - 1) % 6 < 3 ? 0x7fffffff : int(0x80000000));
  }
  __syncthreads();
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int v = pnode[s];
    if (v < c_begin || v >= c_end) continue;
    const SahNode nd = nodes[v];
    const uint32_t t = order[s];
    const float4 l = tlo[t], h = thi[t];
    const float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
    int* nb = sb + (v - c_begin) * (3 * kSahBins * kBinWords);
    for (int a = 0; a < 3; ++a) {
      const float lo = comp(nd.clo, a), ext = comp(nd.chi, a) - lo;
      if (!(ext > 0.f)) continue;
      int* w = nb + (a * kSahBins + sah_bin(c[a], lo, ext)) * kBinWords;
      atomicAdd(w, 1);
      atomicMin(w + 1, f2o(l.x)); atomicMin(w + 2, f2o(l.y)); atomicMin(w + 3, f2o(l.z));
      atomicMax(w + 4, f2o(h.x)); atomicMax(w + 5, f2o(h.y)); atomicMax(w + 6, f2o(h.z));
      atomicMin(w + 7, f2o(c[0])); atomicMin(w + 8, f2o(c[1])); atomicMin(w + 9, f2o(c[2]));
      atomicMax(w + 10, f2o(c[0])); atomicMax(w + 11, f2o(c[1])); atomicMax(w + 12, f2o(c[2]));
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
    const int* w = sb + b * kBinWords;
    if (!w[0]) continue;
    int* g = bins + size_t(b) * kBinWords;
    atomicAdd(g, w[0]);
    for (int k = 1; k < kBinWords; ++k) {
      if ((k - 1) % 6 < 3) atomicMin(g + k, w[k]);
      else atomicMax(g + k, w[k]);
    }
  }
}

// 2. decision per open node of one chunk [c_begin, c_end) of the level:
// split[v - lvl_begin] = {axis (-1: leaf, 3: median), bin, left count}, and
// for a split the two children's boxes (from the bins on each side of the
// plane; a median split keeps the parent's boxes) in kids[2 (v - lvl_begin)].
__global__ void k_sah_split(const SahNode* __restrict__ nodes, int lvl_begin, int c_begin, int c_end,
                            const int* __restrict__ bins, int4* __restrict__ split, SahNode* __restrict__ kids,
                            int* __restrict__ nkids) {
  const int v = c_begin + int(blockIdx.x * blockDim.x + threadIdx.x);
  if (v >= c_end) return;
  const SahNode nd = nodes[v];
  const int n = nd.end - nd.begin;
  const int* nb = bins + size_t(v - c_begin) * (3 * kSahBins * kBinWords);
  int best_axis = -1, best_split = -1, best_left = 0;
  float best_cost = 3.402823466e38f;
  if (n > 1 && nd.depth < kSahMaxDepth) {
    for (int a = 0; a < 3; ++a) {
      if (!(comp(nd.chi, a) - comp(nd.clo, a) > 0.f)) continue;
      const int* ab = nb + a * kSahBins * kBinWords;
      float right_area[kSahBins];
      int right_cnt[kSahBins];
      float lx = 3.402823466e38f, ly = lx, lz = lx, hx = -lx, hy = -lx, hz = -lx;
      int cnt = 0;
      for (int b = kSahBins - 1; b > 0; --b) {
        const int* w = ab + b * kBinWords;
        if (w[0]) {
          lx = fminf(lx, o2f(w[1])); ly = fminf(ly, o2f(w[2])); lz = fminf(lz, o2f(w[3]));
          hx = fmaxf(hx, o2f(w[4])); hy = fmaxf(hy, o2f(w[5])); hz = fmaxf(hz, o2f(w[6]));
        }
        cnt += w[0];
        right_area[b] = sah_area(lx, ly, lz, hx, hy, hz);
        right_cnt[b] = cnt;
      }
      lx = 3.402823466e38f; ly = lx; lz = lx; hx = -lx; hy = -lx; hz = -lx;
      cnt = 0;
      for (int b = 0; b < kSahBins - 1; ++b) {
        const int* w = ab + b * kBinWords;
        if (w[0]) {
          lx = fminf(lx, o2f(w[1])); ly = fminf(ly, o2f(w[2])); lz = fminf(lz, o2f(w[3]));
          hx = fmaxf(hx, o2f(w[4])); hy = fmaxf(hy, o2f(w[5])); hz = fmaxf(hz, o2f(w[6]));
        }
        cnt += w[0];
        if (cnt == 0 || right_cnt[b + 1] == 0) continue;
        const float cost = __fadd_rn(__fmul_rn(sah_area(lx, ly, lz, hx, hy, hz), float(cnt)),
                                     __fmul_rn(right_area[b + 1], float(right_cnt[b + 1])));
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = a;
          best_split = b;
          best_left = cnt;
        }
      }
    }
    const float area = sah_area(nd.lo.x, nd.lo.y, nd.lo.z, nd.hi.x, nd.hi.y, nd.hi.z);
    if (best_axis < 0) {
      if (n > kSahMaxLeaf) {  // coincident centroids: halve the range
        best_axis = 3;
        best_left = n / 2;
      }
    } else if (n <= kSahMaxLeaf && __fmul_rn(area, float(n)) <= __fadd_rn(area, best_cost)) {
      best_axis = -1;
    }
  }
  const int k = v - lvl_begin;
  split[k] = make_int4(best_axis, best_split, best_left, 0);
  nkids[k] = best_axis >= 0 ? 2 : 0;
  if (best_axis < 0) return;
  SahNode L = nd, R = nd;
  L.depth = R.depth = nd.depth + 1;
  L.end = nd.begin + best_left;
  R.begin = L.end;
  if (best_axis < 3) {
    const int* ab = nb + best_axis * kSahBins * kBinWords;
    float b[2][12];
    for (int side = 0; side < 2; ++side)
      for (int j = 0; j < 12; ++j) b[side][j] = (j % 6) < 3 ? 3.402823466e38f : -3.402823466e38f;
    for (int bin = 0; bin < kSahBins; ++bin) {
      const int* w = ab + bin * kBinWords;
      if (!w[0]) continue;
      float* d = b[bin <= best_split ? 0 : 1];
      for (int j = 0; j < 12; ++j) d[j] = (j % 6) < 3 ? fminf(d[j], o2f(w[1 + j])) : fmaxf(d[j], o2f(w[1 + j]));
    }
    SahNode* c[2] = {&L, &R};
    for (int side = 0; side < 2; ++side) {
      const float* d = b[side];
      c[side]->lo = make_float4(d[0], d[1], d[2], 0.f);
      c[side]->hi = make_float4(d[3], d[4], d[5], 0.f);
      c[side]->clo = make_float4(d[6], d[7], d[8], 0.f);
      c[side]->chi = make_float4(d[9], d[10], d[11], 0.f);
    }
  }
  kids[2 * k] = L;
  kids[2 * k + 1] = R;
}

// 3. child records and this level's node records (reference layout)
__global__ void k_sah_children(SahNode* __restrict__ nodes, int lvl_begin, int lvl_end, const int4* __restrict__ split,
                               const SahNode* __restrict__ kids, const int* __restrict__ kid_base, int next_begin,
                               float4* __restrict__ out) {
  const int v = lvl_begin + int(blockIdx.x * blockDim.x + threadIdx.x);
  if (v >= lvl_end) return;
  const int k = v - lvl_begin;
  const SahNode nd = nodes[v];
  float4* o = out + 4 * size_t(v);
  if (split[k].x < 0) {
    o[0] = make_float4(0.f, 0.f, 0.f, ibits(0));
    o[1] = make_float4(0.f, 0.f, 0.f, ibits(0));
    o[2] = make_float4(0.f, 0.f, 0.f, ibits(nd.end - nd.begin));
    o[3] = make_float4(0.f, 0.f, 0.f, ibits(nd.begin));
    return;
  }
  const int left = next_begin + kid_base[k], right = left + 1;
  const SahNode L = kids[2 * k], R = kids[2 * k + 1];
  nodes[left] = L;
  nodes[right] = R;
  o[0] = make_float4(L.lo.x, L.lo.y, L.lo.z, ibits(left));
  o[1] = make_float4(L.hi.x, L.hi.y, L.hi.z, ibits(right));
  o[2] = make_float4(R.lo.x, R.lo.y, R.lo.z, ibits(0));
  o[3] = make_float4(R.hi.x, R.hi.y, R.hi.z, ibits(0));
}

// 4a. goes-left flags of the slots of split nodes (0 elsewhere)
__global__ void k_sah_flags(uint32_t n, const uint32_t* __restrict__ order, const int* __restrict__ pnode,
                            const float4* __restrict__ tlo, const float4* __restrict__ thi,
                            const SahNode* __restrict__ nodes, int lvl_begin, int lvl_end,
                            const int4* __restrict__ split, int* __restrict__ flag) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int v = pnode[s];
    int f = 0;
    if (v >= lvl_begin && v < lvl_end) {
      const int4 sp = split[v - lvl_begin];
      if (sp.x == 3) {
        f = int(s) < nodes[v].begin + sp.z ? 1 : 0;
      } else if (sp.x >= 0) {
        const SahNode nd = nodes[v];
        const uint32_t t = order[s];
        const float4 l = tlo[t], h = thi[t];
        const float c = sp.x == 0 ? 0.5f * (l.x + h.x) : (sp.x == 1 ? 0.5f * (l.y + h.y) : 0.5f * (l.z + h.z));
        const float lo = comp(nd.clo, sp.x), ext = comp(nd.chi, sp.x) - lo;
        f = sah_bin(c, lo, ext) <= sp.y ? 1 : 0;
      }
    }
    flag[s] = f;
  }
}

// 4b. stable partition: left slots keep their order at the front of the
// range, right slots after them; slots of leaves stay
__global__ void k_sah_scatter(uint32_t n, const uint32_t* __restrict__ order, const int* __restrict__ pnode,
                              const SahNode* __restrict__ nodes, int lvl_begin, int lvl_end,
                              const int4* __restrict__ split, const int* __restrict__ kid_base, int next_begin,
                              const int* __restrict__ flag, const int* __restrict__ scan,
                              uint32_t* __restrict__ order2, int* __restrict__ pnode2, int* __restrict__ err) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int v = pnode[s];
    uint32_t dst = s;
    int nv = v;
    if (v >= lvl_begin && v < lvl_end) {
      const int4 sp = split[v - lvl_begin];
      if (sp.x >= 0) {
        const int b = nodes[v].begin;
        const int left_before = scan[s] - scan[b];  // goes-left slots in [b, s)
        const int left = next_begin + kid_base[v - lvl_begin];
        if (flag[s]) {
          dst = uint32_t(b + left_before);
          nv = left;
        } else {
          dst = uint32_t(b + sp.z + (int(s) - b - left_before));
          nv = left + 1;
        }
      }
    }
    if (dst >= n) {  // a left count that disagrees with the flags: reported, never written
      atomicExch(err, 1);
      continue;
    }
    order2[dst] = order[s];
    pnode2[dst] = nv;
  }
}

__global__ void k_sah_root(uint32_t n, const float* __restrict__ block_bounds, int nblocks, SahNode* __restrict__ root,
                           uint32_t* __restrict__ order, int* __restrict__ pnode) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float cb[6] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f, -3.402823466e38f, -3.402823466e38f,
                   -3.402823466e38f};
    for (int b = 0; b < nblocks; ++b)
      for (int k = 0; k < 6; ++k)
        cb[k] = k < 3 ? fminf(cb[k], block_bounds[6 * b + k]) : fmaxf(cb[k], block_bounds[6 * b + k]);
    SahNode r{};
    r.clo = make_float4(cb[0], cb[1], cb[2], 0.f);
    r.chi = make_float4(cb[3], cb[4], cb[5], 0.f);
    r.begin = 0;
    r.end = int(n);
    r.depth = 0;
    *root = r;
  }
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    order[t] = t;
    pnode[t] = 0;
  }
}

// the root's box: a reduction over the triangle boxes
__global__ void k_sah_root_box(uint32_t n, const float4* __restrict__ tlo, const float4* __restrict__ thi,
                               int* __restrict__ box) {
  int l[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, h[3] = {int(0x80000000), int(0x80000000), int(0x80000000)};
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const float4 a = tlo[t], b = thi[t];
    l[0] = min(l[0], f2o(a.x)); l[1] = min(l[1], f2o(a.y)); l[2] = min(l[2], f2o(a.z));
    h[0] = max(h[0], f2o(b.x)); h[1] = max(h[1], f2o(b.y)); h[2] = max(h[2], f2o(b.z));
  }
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      l[k] = min(l[k], __shfl_xor_sync(0xffffffffu, l[k], o));
      h[k] = max(h[k], __shfl_xor_sync(0xffffffffu, h[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k) {
      atomicMin(box + k, l[k]);
      atomicMax(box + 3 + k, h[k]);
    }
}

__global__ void k_sah_root_set(SahNode* root, const int* __restrict__ box) {
  if (threadIdx.x == 0) {
    root->lo = make_float4(o2f(box[0]), o2f(box[1]), o2f(box[2]), 0.f);
    root->hi = make_float4(o2f(box[3]), o2f(box[4]), o2f(box[5]), 0.f);
  }
}

__global__ void k_sah_remap(uint32_t n, const uint32_t* __restrict__ order, int32_t* __restrict__ remap) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
    remap[s] = int32_t(order[s]);
}

int build_bvh_device_sah(const float4* verts, const uint32_t* indices, uint32_t ntris, cudaStream_t st,
                         DeviceBvh* out, Status& s) {
  if (ntris == 0) return s.fail(DSPBR_ERR_INVALID, "device BVH: no triangles");
  if (ntris > (1u << 28)) return s.fail(DSPBR_ERR_INVALID, "device BVH: too many triangles");
  const uint32_t n = ntris;
  const size_t cap = 2 * size_t(n) - 1;  // every split leaves both sides non-empty
  constexpr int kChunk = 1 << 16;        // nodes binned per pass (bins: 2.5 KB per node)
  DevBuf<float4> tlo, thi;
  DevBuf<float> bb;
  DevBuf<uint32_t> order, order2;
  DevBuf<int> pnode, pnode2, flag, scan, bins, nkids, kid_base, box, err;
  DevBuf<SahNode> nodes, kids;
  DevBuf<int4> split;
  DevBuf<unsigned char> tmp;
  const int nb = grid(n, 256, 148 * 4);
  TRY_CUDA(s, tlo.alloc(n), "device BVH");
  TRY_CUDA(s, thi.alloc(n), "device BVH");
  TRY_CUDA(s, bb.alloc(6 * size_t(nb)), "device BVH");
  TRY_CUDA(s, order.alloc(n), "device BVH");
  TRY_CUDA(s, order2.alloc(n), "device BVH");
  TRY_CUDA(s, pnode.alloc(n), "device BVH");
  TRY_CUDA(s, pnode2.alloc(n), "device BVH");
  TRY_CUDA(s, flag.alloc(n), "device BVH");
  TRY_CUDA(s, scan.alloc(n), "device BVH");
  TRY_CUDA(s, nodes.alloc(cap), "device BVH");
  TRY_CUDA(s, box.alloc(6), "device BVH");
  TRY_CUDA(s, err.alloc(1), "device BVH");
  TRY_CUDA(s, cudaMemsetAsync(err.p, 0, sizeof(int), st), "device BVH");
  TRY_CUDA(s, bins.alloc(size_t(std::min<size_t>(cap, kChunk)) * 3 * kSahBins * kBinWords), "device BVH");
  TRY_CUDA(s, out->nodes.alloc(cap * 4), "device BVH");
  TRY_CUDA(s, out->remap.alloc(n), "device BVH");
  size_t scan_temp = 0, t2 = 0;
  TRY_CUDA(s, cub::DeviceScan::ExclusiveSum(nullptr, scan_temp, flag.p, scan.p, int(n), st), "device BVH scan");
  TRY_CUDA(s, cub::DeviceScan::ExclusiveSum(nullptr, t2, nkids.p, kid_base.p, int(n) + 1, st), "device BVH scan");
  scan_temp = std::max(scan_temp, t2);
  TRY_CUDA(s, tmp.alloc(std::max<size_t>(scan_temp, 1)), "device BVH");
  TRY_CUDA(s, cudaFuncSetAttribute(k_sah_bin_shared, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kSharedBinNodes * 3 * kSahBins * kBinWords * int(sizeof(int))),
           "device BVH");
  k_tri_bounds<<<nb, 256, 0, st>>>(verts, indices, n, tlo.p, thi.p, bb.p);
  k_sah_root<<<grid(n, 256, 148 * 8), 256, 0, st>>>(n, bb.p, nb, nodes.p, order.p, pnode.p);
  const int box_init[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, int(0x80000000), int(0x80000000), int(0x80000000)};
  TRY_CUDA(s, cudaMemcpyAsync(box.p, box_init, sizeof box_init, cudaMemcpyHostToDevice, st), "device BVH");
  k_sah_root_box<<<grid(n, 256, 148 * 8), 256, 0, st>>>(n, tlo.p, thi.p, box.p);
  k_sah_root_set<<<1, 32, 0, st>>>(nodes.p, box.p);
  TRY_CUDA(s, cudaGetLastError(), "device BVH");
  int lvl_begin = 0, lvl_end = 1;
  size_t level_cap = 0;
  while (lvl_end > lvl_begin) {
    const int width = lvl_end - lvl_begin;
    if (size_t(width) > level_cap) {
      level_cap = std::max<size_t>(size_t(width), 2 * level_cap);
      TRY_CUDA(s, split.alloc(level_cap), "device BVH");
      TRY_CUDA(s, kids.alloc(2 * level_cap), "device BVH");
      TRY_CUDA(s, nkids.alloc(level_cap + 1), "device BVH");
      TRY_CUDA(s, kid_base.alloc(level_cap + 1), "device BVH");
    }
    for (int c_begin = lvl_begin; c_begin < lvl_end; c_begin += kChunk) {
      const int c_end = std::min(lvl_end, c_begin + kChunk);
      const uint32_t words = uint32_t(c_end - c_begin) * 3u * kSahBins * kBinWords;
      k_sah_init<<<grid(words, 256, 148 * 8), 256, 0, st>>>(n, bins.p, words);
      if (c_end - c_begin <= kSharedBinNodes) {
        const size_t smem = size_t(words) * sizeof(int);
        k_sah_bin_shared<<<grid(n, 256, 148 * 2), 256, smem, st>>>(n, order.p, pnode.p, tlo.p, thi.p, nodes.p,
                                                                   c_begin, c_end, bins.p);
      } else {
        k_sah_bin<<<grid(n, 256, 148 * 8), 256, 0, st>>>(n, order.p, pnode.p, tlo.p, thi.p, nodes.p, c_begin, c_end,
                                                         bins.p);
      }
      k_sah_split<<<(c_end - c_begin + 127) / 128, 128, 0, st>>>(nodes.p, lvl_begin, c_begin, c_end, bins.p,
                                                                 split.p, kids.p, nkids.p);
    }
    TRY_CUDA(s, cudaMemsetAsync(nkids.p + width, 0, sizeof(int), st), "device BVH");
    TRY_CUDA(s, cub::DeviceScan::ExclusiveSum(tmp.p, scan_temp, nkids.p, kid_base.p, width + 1, st),
             "device BVH scan");
    int total_kids = 0;
    TRY_CUDA(s, cudaMemcpyAsync(&total_kids, kid_base.p + width, sizeof(int), cudaMemcpyDeviceToHost, st),
             "device BVH");
    TRY_CUDA(s, cudaStreamSynchronize(st), "device BVH");
    if (size_t(lvl_end) + size_t(total_kids) > cap) return s.fail(DSPBR_ERR_DEVICE_FAULT, "device BVH: node overflow");
    k_sah_children<<<(width + 127) / 128, 128, 0, st>>>(nodes.p, lvl_begin, lvl_end, split.p, kids.p, kid_base.p,
                                                        lvl_end, out->nodes.p);
    if (total_kids > 0) {
      k_sah_flags<<<grid(n, 256, 148 * 8), 256, 0, st>>>(n, order.p, pnode.p, tlo.p, thi.p, nodes.p, lvl_begin,
                                                         lvl_end, split.p, flag.p);
      TRY_CUDA(s, cub::DeviceScan::ExclusiveSum(tmp.p, scan_temp, flag.p, scan.p, int(n), st), "device BVH scan");
      k_sah_scatter<<<grid(n, 256, 148 * 8), 256, 0, st>>>(n, order.p, pnode.p, nodes.p, lvl_begin, lvl_end, split.p,
                                                           kid_base.p, lvl_end, flag.p, scan.p, order2.p, pnode2.p,
                                                           err.p);
      order.swap(order2);
      pnode.swap(pnode2);
    }
    TRY_CUDA(s, cudaGetLastError(), "device BVH");
    lvl_begin = lvl_end;
    lvl_end += total_kids;
  }
  k_sah_remap<<<grid(n, 256, 148 * 8), 256, 0, st>>>(n, order.p, out->remap.p);
  TRY_CUDA(s, cudaGetLastError(), "device BVH");
  int bad = 0;
  TRY_CUDA(s, cudaMemcpyAsync(&bad, err.p, sizeof(int), cudaMemcpyDeviceToHost, st), "device BVH");
  // the temporaries are freed at return: wait for the kernels that use them
  TRY_CUDA(s, cudaStreamSynchronize(st), "device BVH");
  if (bad) return s.fail(DSPBR_ERR_DEVICE_FAULT, "device BVH: partition counts disagree");
  out->num_nodes = uint32_t(lvl_end);
  out->num_slots = n;
  return DSPBR_OK;
}

int collapse_bvh4_device(const DeviceBvh& bin, cudaStream_t st, DeviceWideBvh* out, Status& s) {
  const uint32_t nn = bin.num_nodes;
  if (nn == 0) return s.fail(DSPBR_ERR_INVALID, "wide BVH: empty tree");
  // the root: a leaf root is tested without a box; otherwise wide node 0
  int32_t root_cnt = 0, root_first = 0;
  TRY_CUDA(s, cudaMemcpyAsync(&root_cnt, reinterpret_cast<const char*>(bin.nodes.p) + 44, 4, cudaMemcpyDeviceToHost, st),
           "wide BVH");
  TRY_CUDA(s, cudaMemcpyAsync(&root_first, reinterpret_cast<const char*>(bin.nodes.p) + 60, 4, cudaMemcpyDeviceToHost,
                              st), "wide BVH");
  TRY_CUDA(s, cudaStreamSynchronize(st), "wide BVH");
  TRY_CUDA(s, out->leaves.alloc(nn), "wide BVH");
  if (root_cnt > 0) {
    long long b0 = root_first > 0 ? root_first : 0;
    long long b1 = (long long)root_first + (root_cnt < 64 ? root_cnt : 64);
    if (b1 > (long long)bin.num_slots) b1 = bin.num_slots;
    if (b1 < b0) b1 = b0;
    int2 lf = make_int2(int(b0), int(b1));
    TRY_CUDA(s, cudaMemcpyAsync(out->leaves.p, &lf, sizeof lf, cudaMemcpyHostToDevice, st), "wide BVH");
    TRY_CUDA(s, out->nodes.alloc(8), "wide BVH");
    TRY_CUDA(s, cudaStreamSynchronize(st), "wide BVH");
    out->root = ~0;
    out->num_nodes = 0;
    out->num_leaves = 1;
    return DSPBR_OK;
  }
  // each wide node holds >= 2 children, so there are fewer wide nodes than binary inner nodes
  TRY_CUDA(s, out->nodes.alloc(size_t(nn) * 8), "wide BVH");
  DevBuf<int2> fa, fb;
  DevBuf<WideCounters> ctr;
  TRY_CUDA(s, fa.alloc(nn), "wide BVH");
  TRY_CUDA(s, fb.alloc(nn), "wide BVH");
  TRY_CUDA(s, ctr.alloc(1), "wide BVH");
  WideCounters h{1, 0, 0};  // wide node 0 is the root
  int2 first = make_int2(0, 0);
  TRY_CUDA(s, cudaMemcpyAsync(ctr.p, &h, sizeof h, cudaMemcpyHostToDevice, st), "wide BVH");
  TRY_CUDA(s, cudaMemcpyAsync(fa.p, &first, sizeof first, cudaMemcpyHostToDevice, st), "wide BVH");
  int count = 1;
  int2* cur = fa.p;
  int2* nxt = fb.p;
  for (uint32_t level = 0; count > 0 && level <= nn; ++level) {
    TRY_CUDA(s, cudaMemsetAsync(&ctr.p->next, 0, sizeof(int), st), "wide BVH");
    k_collapse_level<<<grid(count, 128, 148 * 8), 128, 0, st>>>(bin.nodes.p, nn, bin.num_slots, cur, count, nxt,
                                                               out->nodes.p, out->leaves.p, ctr.p);
    TRY_CUDA(s, cudaGetLastError(), "wide BVH");
    TRY_CUDA(s, cudaMemcpyAsync(&h, ctr.p, sizeof h, cudaMemcpyDeviceToHost, st), "wide BVH");
    TRY_CUDA(s, cudaStreamSynchronize(st), "wide BVH");
    count = h.next;
    std::swap(cur, nxt);
  }
  if (count != 0) return s.fail(DSPBR_ERR_INVALID, "wide BVH: the tree does not end (cyclic input)");
  out->root = 0;
  out->num_nodes = uint32_t(h.nodes);
  out->num_leaves = uint32_t(h.leaves);
  return DSPBR_OK;
}

int build_cw8_device(const float4* bin, uint32_t nn, uint32_t num_slots, const float4* tris, cudaStream_t st,
                     DeviceCw8* out, Status& s) {
  out->nodes.reset();
  out->recs.reset();
  out->num_nodes = out->num_recs = out->levels = 0;
  if (nn == 0) return DSPBR_OK;
  int32_t root_cnt = 0;
  TRY_CUDA(s, cudaMemcpyAsync(&root_cnt, reinterpret_cast<const char*>(bin) + 44, 4, cudaMemcpyDeviceToHost, st),
           "8-wide BVH");
  DevBuf<unsigned long long> total;
  TRY_CUDA(s, total.alloc(1), "8-wide BVH");
  TRY_CUDA(s, cudaMemsetAsync(total.p, 0, sizeof(unsigned long long), st), "8-wide BVH");
  k_cw8_count<<<grid(nn, 256, 148 * 8), 256, 0, st>>>(bin, nn, num_slots, total.p);
  TRY_CUDA(s, cudaGetLastError(), "8-wide BVH");
  unsigned long long nrec = 0;
  TRY_CUDA(s, cudaMemcpyAsync(&nrec, total.p, sizeof nrec, cudaMemcpyDeviceToHost, st), "8-wide BVH");
  TRY_CUDA(s, cudaStreamSynchronize(st), "8-wide BVH");
  // a leaf root has no box to quantise, and record indices are int: the 4-wide tree serves those
  if (root_cnt > 0 || nrec == 0 || nrec > 0x7fffffffull / 3) return DSPBR_OK;
  DevBuf<uint4> nodes;
  DevBuf<float4> recs;
  DevBuf<int32_t> src;
  DevBuf<int2> fa, fb;
  DevBuf<Cw8Counters> ctr;
  TRY_CUDA(s, nodes.alloc(size_t(nn) * 5), "8-wide BVH");
  TRY_CUDA(s, recs.alloc(size_t(nrec) * 3), "8-wide BVH");
  TRY_CUDA(s, src.alloc(nrec), "8-wide BVH");
  TRY_CUDA(s, fa.alloc(nn), "8-wide BVH");
  TRY_CUDA(s, fb.alloc(nn), "8-wide BVH");
  TRY_CUDA(s, ctr.alloc(1), "8-wide BVH");
  Cw8Counters h{1, 0, 0, 0};  // node 0 is the root
  int2 first = make_int2(0, 0);
  TRY_CUDA(s, cudaMemcpyAsync(ctr.p, &h, sizeof h, cudaMemcpyHostToDevice, st), "8-wide BVH");
  TRY_CUDA(s, cudaMemcpyAsync(fa.p, &first, sizeof first, cudaMemcpyHostToDevice, st), "8-wide BVH");
  int count = 1;
  uint32_t levels = 0;
  int2* cur = fa.p;
  int2* nxt = fb.p;
  for (; count > 0 && levels <= nn; ++levels) {
    TRY_CUDA(s, cudaMemsetAsync(&ctr.p->next, 0, sizeof(int), st), "8-wide BVH");
    k_cw8_level<<<grid(count, 64, 148 * 16), 64, 0, st>>>(bin, nn, num_slots, cur, count, nxt, int(nn), nodes.p,
                                                          int(nn), recs.p, src.p, int(nrec), ctr.p);
    TRY_CUDA(s, cudaGetLastError(), "8-wide BVH");
    TRY_CUDA(s, cudaMemcpyAsync(&h, ctr.p, sizeof h, cudaMemcpyDeviceToHost, st), "8-wide BVH");
    TRY_CUDA(s, cudaStreamSynchronize(st), "8-wide BVH");
    if (h.error) return DSPBR_OK;  // an axis no frame fits, or a malformed tree: the 4-wide tree serves
    count = std::min(h.next, int(nn));
    std::swap(cur, nxt);
  }
  if (count != 0) return DSPBR_OK;
  k_cw8_gather<<<grid(size_t(h.recs), 256, 148 * 8), 256, 0, st>>>(src.p, h.recs, tris, recs.p);
  TRY_CUDA(s, cudaGetLastError(), "8-wide BVH");
  TRY_CUDA(s, out->nodes.alloc(size_t(h.nodes) * 5), "8-wide BVH");
  TRY_CUDA(s, cudaMemcpyAsync(out->nodes.p, nodes.p, size_t(h.nodes) * 5 * sizeof(uint4), cudaMemcpyDeviceToDevice, st),
           "8-wide BVH");
  TRY_CUDA(s, cudaStreamSynchronize(st), "8-wide BVH");
  out->recs.swap(recs);
  out->num_nodes = uint32_t(h.nodes);
  out->num_recs = uint32_t(h.recs);
  out->levels = levels;
  return DSPBR_OK;
}

}  // namespace dspbr
