// Device-side scene/IBL views, traversal, RNG, camera and hit set-up.
#pragma once
#include <stdint.h>

#include "material.cuh"
#include "vecmath.cuh"

namespace dspbr {

// reference constants (constants.glsl:12-21, bvh.glsl:8-10)
constexpr float kGlslPi = 3.14159265358979323f;
constexpr float kGlslTwoPi = 6.28318530717958648f;
constexpr float kEps = 1e-8f;
constexpr float kEpsCos = 0.001f;
constexpr float kEpsPdf = 0.001f;
constexpr float kTfarMax = 100000.0f;
constexpr float kBvhFar = 1e30f;
constexpr int kStackSize = 64;
constexpr int kMaxSteps = 4096;
constexpr int kMaxLeafTris = 64;

// Device scene.  nodes: 4 float4 per node, child index / count / first are
// stored as int bits in .w (converted once from the reference's floats with the
// same truncating conversion the shader's int() performs).  tris: 3 float4 per
// BVH leaf slot, pre-gathered in leaf order: (p0.xyz, mesh triangle id bits),
// (p1 - p0, 0), (p2 - p0, 0); id -1 marks a remap entry the reference skips.
// One RGBA8 texture array (all layers share a resolution; scene_data_webgl2.ts:266-300).
struct DevTexArray {
  const uchar4* __restrict__ data;  // layers x h x w
  int w, h, layers;
};

struct DevScene {
  const float4* __restrict__ nodes;
  const float4* __restrict__ tris;
  const float4* __restrict__ verts;      // 5 float4 per vertex (20-float record)
  const uint32_t* __restrict__ indices;  // 3 per triangle
  const float4* __restrict__ materials;  // 17 float4 per material (68 floats)
  const uint8_t* __restrict__ tri_class;  // shading class per mesh triangle
  const float4* __restrict__ wnodes;      // 4-wide BVH: 8 float4 per node (bvh_wide.h WideNode4)
  const int2* __restrict__ wleaves;       // leaf-slot range [x, y) per wide leaf
  int wroot;                              // >= 0: wide node; < 0: ~leaf (the binary root is a leaf)
  const uint4* __restrict__ cnodes;       // compressed 8-wide BVH (5 uint4 per node), or null
  const float4* __restrict__ ctris;       // its leaf records: header (exact box, count) + triangle records
  int num_nodes, num_slots, num_tris, num_materials;
  int boxes_finite;  // every node bound is finite (checked at upload)
  int wide;          // closest-hit / any-hit queries of paths use the wide BVH
  const float4* __restrict__ texinfo;         // 2 float4 per TexInfo (material.ts:483-523)
  const DevTexArray* __restrict__ tex_arrays;
  int num_texinfo, num_tex_arrays;
};

struct DevIbl {
  const float4* __restrict__ rgba;  // w*h, row 0 = v 0 (zenith)
  const float* __restrict__ pdf;    // w*h  (renderer.ts:802-838 tables)
  const float* __restrict__ cdf;
  const float* __restrict__ ypdf;   // h
  const float* __restrict__ ycdf;
  const float* __restrict__ alias_prob;  // w*h
  const int* __restrict__ alias_idx;
  int w, h;
};

// ---- RNG ----------------------------------------------------------------------
// George Marsaglia MWC of rng.glsl:5-29, seeded from the fragment coordinate.
struct Mwc {
  uint32_t x, y;
};
DEV Mwc mwc_init(int seed, int px, int py) {
  float off = float(seed * 17);
  float fx = __fadd_rn(float(px), 0.5f), fy = __fadd_rn(float(py), 0.5f);
  Mwc s;
  s.x = __float2uint_rz(__fmul_rn(397.6432f, __fadd_rn(fx, off)));
  s.y = __float2uint_rz(__fmul_rn(397.6432f, __fadd_rn(fy, 0.0f)));
  s.x ^= __float2uint_rz(__fmul_rn(32.9875f, __fadd_rn(fy, off)));
  s.y ^= __float2uint_rz(__fmul_rn(32.9875f, __fadd_rn(fx, 0.0f)));
  return s;
}
DEV float mwc_float(Mwc& s) {
  s.x = 36969u * (s.x & 65535u) + (s.x >> 16u);
  s.y = 18000u * (s.y & 65535u) + (s.y >> 16u);
  uint32_t r = (s.x << 16u) + s.y;
  return __fdiv_rn(__uint2float_rn(r), 4294967296.0f);
}

// PCG32 (O'Neill, XSH-RR output), one stream per pixel sample.  State is the
// 64-bit LCG state; the stream increment is derived from the stream id.
DEV uint64_t pcg_inc(uint64_t stream) { return (stream << 1u) | 1u; }
DEV uint32_t pcg_next(uint64_t& state, uint64_t inc) {
  uint64_t old = state;
  state = old * 6364136223846793005ull + inc;
  uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
  uint32_t rot = uint32_t(old >> 59u);
  return (xs >> rot) | (xs << ((32u - rot) & 31u));
}
DEV uint64_t pcg_init(uint64_t seed, uint64_t stream) {
  uint64_t inc = pcg_inc(stream);
  uint64_t st = 0;
  pcg_next(st, inc);
  st += seed;
  pcg_next(st, inc);
  return st;
}
DEV float pcg_float(uint64_t& state, uint64_t inc) { return float(pcg_next(state, inc) >> 8) * (1.0f / 16777216.0f); }

struct Rng {
  uint64_t state;
  uint64_t inc;  // 0 selects MWC (state = x | y << 32)
  DEV float next() {
    if (inc == 0) {
      Mwc m{uint32_t(state), uint32_t(state >> 32)};
      float f = mwc_float(m);
      state = uint64_t(m.x) | (uint64_t(m.y) << 32);
      return f;
    }
    return pcg_float(state, inc);
  }
};

// ---- traversal (bvh.glsl:31-62, 149-229) ------------------------------------------
struct Hit {
  int tri;
  float t, u, v;
};

// bvh_intersect_bounds (bvh.glsl:31-41).  kExactNaN keeps GLSL's min/max
// (y<x ? y : x), which differs from fminf/fmaxf only when an operand is NaN.
// No slab value can be NaN when the ray origin and 1/dir are finite and the
// box bounds are finite; traverse() then takes the FMNMX form, whose decisions
// are identical (a -0/+0 difference does not change any comparison).
template <bool kExactNaN>
DEV float slab(float4 bmin, float4 bmax, v3 org, v3 inv, float tfar) {
  float t0x = __fmul_rn(__fsub_rn(bmin.x, org.x), inv.x), t1x = __fmul_rn(__fsub_rn(bmax.x, org.x), inv.x);
  float t0y = __fmul_rn(__fsub_rn(bmin.y, org.y), inv.y), t1y = __fmul_rn(__fsub_rn(bmax.y, org.y), inv.y);
  float t0z = __fmul_rn(__fsub_rn(bmin.z, org.z), inv.z), t1z = __fmul_rn(__fsub_rn(bmax.z, org.z), inv.z);
  float tmin, tmax;
  if (kExactNaN) {
    tmin = gmax(gmax(gmin(t0x, t1x), gmin(t0y, t1y)), gmin(t0z, t1z));
    tmax = gmin(gmin(gmax(t0x, t1x), gmax(t0y, t1y)), gmax(t0z, t1z));
    if (isnan(tmin) || isnan(tmax)) return kBvhFar;
  } else {
    tmin = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
    tmax = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
  }
  if (tmin > tmax || tmax < 0.f || tmin >= tfar) return kBvhFar;
  return tmin;
}

// Moller-Trumbore with the reference's rejection tests, every operation
// rounded separately (identical to the IEEE host oracle).
DEV bool intersect_tri(v3 org, v3 dir, float4 a, float4 b, float4 c, float tfar, float& t, float& u, float& v) {
  v3 p0 = mk(a), e0 = mk(b), e1 = mk(c);
  v3 pv = cross_rn(dir, e1);
  float det = dot_rn(e0, pv);
  if (fabsf(det) < kEps) return false;
  float f = __fdiv_rn(1.0f, det);
  v3 s = sub_rn(org, p0);
  u = __fmul_rn(f, dot_rn(s, pv));
  if (u < 0.f || u > 1.f) return false;
  v3 q = cross_rn(s, e0);
  v = __fmul_rn(f, dot_rn(dir, q));
  if (v < 0.f || __fadd_rn(u, v) > 1.f) return false;
  t = __fmul_rn(f, dot_rn(e1, q));
  if (t < kEps || t >= tfar) return false;
  return true;
}

DEV v3 inv_dir(v3 d) { return mk(__fdiv_rn(1.f, d.x), __fdiv_rn(1.f, d.y), __fdiv_rn(1.f, d.z)); }

// Stack traversal with the reference's limits: 64-entry stack (pushes beyond
// it are dropped), 4096 steps, 64 triangles per leaf, node-range and
// self-reference checks.  kAny: stop at the first accepted triangle (same
// boolean as the reference's closest-hit isOccluded).  Returns false and sets
// `aborted` when the step cap ends the loop with work left.
template <bool kAny, bool kExactNaN>
DEV bool traverse_impl(const DevScene& s, v3 org, v3 inv, v3 dir, float tfar, Hit& hit, bool& aborted,
                       uint32_t* nodes_visited, uint32_t* tris_tested) {
  hit.t = tfar;
  hit.tri = -1;
  hit.u = hit.v = 0.f;
  int stack[kStackSize];
  int top = 1;
  stack[0] = 0;
  int step = 0;
  for (; step < kMaxSteps && top > 0; ++step) {
    int ni = stack[--top];
    if (ni < 0 || ni >= s.num_nodes) continue;
    if (nodes_visited) ++*nodes_visited;
    const float4* nd = s.nodes + 4 * size_t(ni);
    float4 n0 = __ldg(nd), n1 = __ldg(nd + 1), n2 = __ldg(nd + 2), n3 = __ldg(nd + 3);
    int cnt = __float_as_int(n2.w);
    if (cnt > 0) {
      int first = __float_as_int(n3.w);
      int end = min(first + min(cnt, kMaxLeafTris), s.num_slots);
      for (int i = max(first, 0); i < end; ++i) {
        const float4* tp = s.tris + 3 * size_t(i);
        float4 a = __ldg(tp);
        int id = __float_as_int(a.w);
        if (id < 0) continue;
        if (tris_tested) ++*tris_tested;
        float t, u, v;
        if (intersect_tri(org, dir, a, __ldg(tp + 1), __ldg(tp + 2), hit.t, t, u, v)) {
          hit.t = t; hit.tri = id; hit.u = u; hit.v = v;
          if (kAny) { aborted = false; return true; }
        }
      }
    } else {
      int left = __float_as_int(n0.w), right = __float_as_int(n1.w);
      float d0 = slab<kExactNaN>(n0, n1, org, inv, hit.t);
      float d1 = slab<kExactNaN>(n2, n3, org, inv, hit.t);
      // bvh_push_child (bvh.glsl:141-145): bounded stack, valid node, not self
      auto push = [&](int c) {
        if (top < kStackSize && c >= 0 && c < s.num_nodes && c != ni) stack[top++] = c;
      };
      if (d0 < kBvhFar && d1 < kBvhFar) {
        if (d0 < d1) { push(right); push(left); }
        else { push(left); push(right); }
      } else if (d0 < kBvhFar) {
        push(left);
      } else if (d1 < kBvhFar) {
        push(right);
      }
    }
  }
  aborted = (top > 0 && step >= kMaxSteps);
  return hit.tri >= 0;
}

DEV bool finite3(v3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

// ---- 4-wide traversal ------------------------------------------------------------------
// Same boxes, same slab arithmetic and same triangle test as the binary
// traversal above, over the collapsed 4-wide tree: the children hit by the ray
// are pushed far to near, so the nearest is visited first.  The closest t is
// the same as the binary traversal's; when two triangles hit at exactly the
// same t, the one tested first is kept, and the order of the tests differs.
constexpr int kWideStack = 96;

DEV void cswap(float& da, int& ca, float& db, int& cb) {
  if (db < da) {
    float t = da; da = db; db = t;
    int c = ca; ca = cb; cb = c;
  }
}

// Resumable state of one 4-wide traversal: the traversal is a sequence of
// steps (one node or one leaf each), so a kernel can run rays of different
// lengths side by side and start a new ray in a lane whose ray has finished.
struct WideTrav {
  int cur;        // the entry visited next (kept out of the stack)
  int top, step;
  bool have;      // an entry is left to visit
  bool overflow;  // a push found the stack full
  bool any_hit;   // kAny: a triangle was accepted
};

DEV void wide_begin(WideTrav& w, int root) {
  w.cur = root;
  w.top = 0;
  w.step = 0;
  w.have = true;
  w.overflow = false;
  w.any_hit = false;
}

// One step; returns whether another step is due (entries left, step cap not
// reached, no accepted triangle for an any-hit ray).  `any` is a run-time
// flag so that closest-hit and any-hit rays can share one instruction stream;
// the callers with a constant get the specialised code.
//
// Stack entries carry the entry distance of the child's box.  A closest-hit
// ray pops an inner node only while that distance is below the closest hit
// found so far: every box below the node lies inside its box, so their slab
// entries are at least as far (the rounded slab arithmetic is monotone in the
// planes) and the reference's test `tmin >= tfar` would reject them all.  The
// result is the same; the node's load is saved.  Leaves are always visited
// (a triangle on a box face may round to a t just below the box's entry).
template <bool kExactNaN>
DEV bool wide_step_rt(const float4* __restrict__ wnodes, const int2* __restrict__ wleaves,
                      const float4* __restrict__ tris, v3 org, v3 inv, v3 dir, Hit& hit, WideTrav& w, int2* stack,
                      bool any) {
  const int e = w.cur;
  bool next_in_register = false;
  if (e < 0) {
    const int2 lf = __ldg(wleaves + ~e);
    for (int i = lf.x; i < lf.y; ++i) {
      const float4* tp = tris + 3 * size_t(i);
      float4 a = __ldg(tp);
      int id = __float_as_int(a.w);
      if (id < 0) continue;
      float t, u, v;
      if (intersect_tri(org, dir, a, __ldg(tp + 1), __ldg(tp + 2), hit.t, t, u, v)) {
        hit.t = t; hit.tri = id; hit.u = u; hit.v = v;
        if (any) {
          w.any_hit = true;
          return false;
        }
      }
    }
  } else {
    const float4* nd = wnodes + 8 * size_t(e);
    const float4 lx = __ldg(nd), ly = __ldg(nd + 1), lz = __ldg(nd + 2);
    const float4 hx = __ldg(nd + 3), hy = __ldg(nd + 4), hz = __ldg(nd + 5);
    const int4 ch = __ldg(reinterpret_cast<const int4*>(nd + 6));
    const int n = __ldg(reinterpret_cast<const int*>(nd + 7));
    float d0 = n > 0 ? slab<kExactNaN>(make_float4(lx.x, ly.x, lz.x, 0.f), make_float4(hx.x, hy.x, hz.x, 0.f), org,
                                       inv, hit.t)
                     : kBvhFar;
    float d1 = n > 1 ? slab<kExactNaN>(make_float4(lx.y, ly.y, lz.y, 0.f), make_float4(hx.y, hy.y, hz.y, 0.f), org,
                                       inv, hit.t)
                     : kBvhFar;
    float d2 = n > 2 ? slab<kExactNaN>(make_float4(lx.z, ly.z, lz.z, 0.f), make_float4(hx.z, hy.z, hz.z, 0.f), org,
                                       inv, hit.t)
                     : kBvhFar;
    float d3 = n > 3 ? slab<kExactNaN>(make_float4(lx.w, ly.w, lz.w, 0.f), make_float4(hx.w, hy.w, hz.w, 0.f), org,
                                       inv, hit.t)
                     : kBvhFar;
    int c0 = ch.x, c1 = ch.y, c2 = ch.z, c3 = ch.w;
    // ascending order of entry distance (5-comparator network)
    cswap(d0, c0, d1, c1);
    cswap(d2, c2, d3, c3);
    cswap(d0, c0, d2, c2);
    cswap(d1, c1, d3, c3);
    cswap(d1, c1, d2, c2);
    auto push = [&](float d, int c) {
      if (d < kBvhFar) {
        if (w.top < kWideStack) stack[w.top++] = make_int2(c, __float_as_int(d));
        else w.overflow = true;
      }
    };
    push(d3, c3);
    push(d2, c2);
    push(d1, c1);
    if (d0 < kBvhFar) {  // nearest child next, without a trip through the stack
      w.cur = c0;
      next_in_register = true;
    }
  }
  if (!next_in_register) {
    w.have = false;
    while (w.top > 0) {
      const int2 en = stack[--w.top];
      if (!kExactNaN && !any && en.x >= 0 && __int_as_float(en.y) >= hit.t) continue;
      w.cur = en.x;
      w.have = true;
      break;
    }
  }
  ++w.step;
  return w.have && w.step < kMaxSteps;
}

template <bool kAny, bool kExactNaN>
DEV bool wide_step(const float4* __restrict__ wnodes, const int2* __restrict__ wleaves,
                   const float4* __restrict__ tris, v3 org, v3 inv, v3 dir, Hit& hit, WideTrav& w, int2* stack) {
  return wide_step_rt<kExactNaN>(wnodes, wleaves, tris, org, inv, dir, hit, w, stack, kAny);
}

// `aborted`: the stack overflowed or the step cap ended the traversal with
// entries left (not when kAny accepted a triangle).
DEV bool wide_aborted(const WideTrav& w) { return !w.any_hit && (w.overflow || (w.have && w.step >= kMaxSteps)); }

template <bool kAny, bool kExactNaN>
DEV bool traverse_wide_impl(const DevScene& s, v3 org, v3 inv, v3 dir, float tfar, Hit& hit, bool& aborted) {
  hit.t = tfar;
  hit.tri = -1;
  hit.u = hit.v = 0.f;
  int2 stack[kWideStack];
  WideTrav w;
  wide_begin(w, s.wroot);
  while (wide_step<kAny, kExactNaN>(s.wnodes, s.wleaves, s.tris, org, inv, dir, hit, w, stack)) {
  }
  aborted = wide_aborted(w);
  return kAny ? (w.any_hit || hit.tri >= 0) : hit.tri >= 0;
}

// ---- compressed 8-wide traversal --------------------------------------------------------
// Node (5 x 16 B, bvh_gpu.h Cw8Node): per axis a frame (P_a, exponent e_a) and
// per child one byte for each of its six planes; the plane of byte q is
// fmaf(2^23 + q, 2^e_a, P_a), the float 2^23 + q made by a byte permute.  The
// builder picks every byte so that this plane lies on or outside the child's
// exact box, evaluated with the same fmaf, and the slab below applies the
// reference's arithmetic, (plane - o) * (1/d) with each operation rounded, to
// that plane.  Rounding is monotone, so a quantised slab is never tighter
// than the exact one: every box the reference's test accepts passes here too.
// Leaves keep their exact box in a header record ahead of their triangles;
// it is tested, like the 4-wide traversal's child boxes, against the closest
// hit of the moment the parent node was visited, so the leaves whose
// triangles are tested are those the exact boxes admit.
//
// Order: the nearest child (quantised entry) is visited next from a register,
// the others are pushed with their entry distance (inner nodes; popped only
// while it lies below the closest hit) or with the closest hit at the push
// (leaves).  Rays whose slab arithmetic can produce NaN (a zero direction
// component, a non-finite origin or box) take the reference's binary
// traversal instead.
struct Cw8Trav {
  int cur;         // node index, or ~header index of a leaf
  float cur_tfar;  // a leaf: the closest hit when its parent was visited
  int top, step;
  bool have, overflow, any_hit;
};

DEV float cw8_plane(uint32_t word, uint32_t sel, float scale, float p) {
  return fmaf(__uint_as_float(__byte_perm(word, 0x4B000000u, sel)), scale, p);
}
DEV float cw8_t(uint32_t word, uint32_t sel, float scale, float p, float o, float inv) {
  return __fmul_rn(__fsub_rn(cw8_plane(word, sel, scale, p), o), inv);
}

DEV bool cw8_step(const uint4* __restrict__ cnodes, const float4* __restrict__ ctris, v3 org, v3 inv, v3 dir,
                  Hit& hit, Cw8Trav& w, int2* stack, bool any) {
  bool next_in_register = false;
  if (w.cur < 0) {
    const float4* hp = ctris + 3 * size_t(~w.cur);
    const float4 h0 = __ldg(hp), h1 = __ldg(hp + 1);
    if (slab<false>(h0, h1, org, inv, w.cur_tfar) < kBvhFar) {
      const int n = __float_as_int(h1.w);
      for (int i = 1; i <= n; ++i) {
        const float4* tp = hp + 3 * size_t(i);
        float4 a = __ldg(tp);
        int id = __float_as_int(a.w);
        if (id < 0) continue;
        float t, u, v;
        if (intersect_tri(org, dir, a, __ldg(tp + 1), __ldg(tp + 2), hit.t, t, u, v)) {
          hit.t = t; hit.tri = id; hit.u = u; hit.v = v;
          if (any) {
            w.any_hit = true;
            return false;
          }
        }
      }
    }
  } else {
    const uint4* nd = cnodes + 5 * size_t(w.cur);
    const uint4 q0 = __ldg(nd), q1 = __ldg(nd + 1), q2 = __ldg(nd + 2), q3 = __ldg(nd + 3), q4 = __ldg(nd + 4);
    const float px = __uint_as_float(q0.x), py = __uint_as_float(q0.y), pz = __uint_as_float(q0.z);
    const float sx = __uint_as_float((q0.w & 0xFFu) << 23), sy = __uint_as_float(((q0.w >> 8) & 0xFFu) << 23),
                sz = __uint_as_float(((q0.w >> 16) & 0xFFu) << 23);
    const uint32_t imask = q0.w >> 24;
    // the near and far planes of each axis (low and high bytes by the sign of the direction)
    const bool nx = inv.x < 0.f, ny = inv.y < 0.f, nz = inv.z < 0.f;
    const uint32_t nx0 = nx ? q3.z : q2.x, nx1 = nx ? q3.w : q2.y, fx0 = nx ? q2.x : q3.z, fx1 = nx ? q2.y : q3.w;
    const uint32_t ny0 = ny ? q4.x : q2.z, ny1 = ny ? q4.y : q2.w, fy0 = ny ? q2.z : q4.x, fy1 = ny ? q2.w : q4.y;
    const uint32_t nz0 = nz ? q4.z : q3.x, nz1 = nz ? q4.w : q3.y, fz0 = nz ? q3.x : q4.z, fz1 = nz ? q3.y : q4.w;
    bool have_best = false;
    int2 best = make_int2(0, 0);
    float best_d = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const uint32_t sel = 0x7540u | uint32_t(c & 3);
      const bool hi = c >= 4;
      const float tnx = cw8_t(hi ? nx1 : nx0, sel, sx, px, org.x, inv.x);
      const float tny = cw8_t(hi ? ny1 : ny0, sel, sy, py, org.y, inv.y);
      const float tnz = cw8_t(hi ? nz1 : nz0, sel, sz, pz, org.z, inv.z);
      const float tfx = cw8_t(hi ? fx1 : fx0, sel, sx, px, org.x, inv.x);
      const float tfy = cw8_t(hi ? fy1 : fy0, sel, sy, py, org.y, inv.y);
      const float tfz = cw8_t(hi ? fz1 : fz0, sel, sz, pz, org.z, inv.z);
      const float tmin = fmaxf(fmaxf(tnx, tny), tnz), tmax = fminf(fminf(tfx, tfy), tfz);
      const bool inner = (imask >> c) & 1u;
      const uint32_t meta = (hi ? q1.w : q1.z) >> (8 * (c & 3)) & 0xFFu;
      if (!(tmin > tmax || tmax < 0.f || tmin >= hit.t) && (inner || meta != 0u)) {
        int2 e;
        if (inner) {
          e = make_int2(int(q1.x + __popc(imask & ((1u << c) - 1u))), __float_as_int(tmin));
        } else {
          // records of the leaf children in lower slots come first
          uint32_t before = c == 0 ? 0u : __dp4a(c < 4 ? q1.z & ((1u << (8 * (c & 3))) - 1u) : q1.z, 0x01010101u, 0u);
          if (c > 4) before = __dp4a(q1.w & ((1u << (8 * (c & 3))) - 1u), 0x01010101u, before);
          e = make_int2(~int(q1.y + before), __float_as_int(hit.t));
        }
        int2 push_e = e;
        bool do_push = have_best;
        if (have_best && tmin < best_d) {
          push_e = best;
          best = e;
          best_d = tmin;
        } else if (!have_best) {
          best = e;
          best_d = tmin;
          have_best = true;
        }
        if (do_push) {
          if (w.top < kWideStack) stack[w.top++] = push_e;
          else w.overflow = true;
        }
      }
    }
    if (have_best) {
      w.cur = best.x;
      w.cur_tfar = __int_as_float(best.y);
      next_in_register = true;
    }
  }
  if (!next_in_register) {
    w.have = false;
    while (w.top > 0) {
      const int2 en = stack[--w.top];
      if (!any && en.x >= 0 && __int_as_float(en.y) >= hit.t) continue;
      w.cur = en.x;
      w.cur_tfar = __int_as_float(en.y);
      w.have = true;
      break;
    }
  }
  ++w.step;
  return w.have && w.step < kMaxSteps;
}

// The compressed 8-wide traversal of one ray (any: stop at the first accepted
// triangle).  Same closest t as the binary traversal except for ties within
// rounding between coplanar faces (two triangles whose t differ by an ulp:
// which is found depends on the visiting order, as in the reference itself).
DEV bool traverse_cw8_rt(const DevScene& s, v3 org, v3 dir, float tfar, bool any, Hit& hit, bool& aborted) {
  v3 inv = inv_dir(dir);
  if (!(s.boxes_finite && finite3(org) && finite3(inv))) {
    bool r = any ? traverse_impl<true, true>(s, org, inv, dir, tfar, hit, aborted, nullptr, nullptr)
                 : traverse_impl<false, true>(s, org, inv, dir, tfar, hit, aborted, nullptr, nullptr);
    return r;
  }
  hit.t = tfar;
  hit.tri = -1;
  hit.u = hit.v = 0.f;
  int2 stack[kWideStack];
  Cw8Trav w{0, tfar, 0, 0, true, false, false};
  while (cw8_step(s.cnodes, s.ctris, org, inv, dir, hit, w, stack, any)) {
  }
  aborted = !w.any_hit && (w.overflow || (w.have && w.step >= kMaxSteps));
  return w.any_hit || hit.tri >= 0;
}

// closest hit (any = false) or any hit (any = true) chosen at run time
DEV bool traverse_wide_rt(const DevScene& s, v3 org, v3 dir, float tfar, bool any, Hit& hit, bool& aborted) {
  if (s.cnodes) return traverse_cw8_rt(s, org, dir, tfar, any, hit, aborted);
  v3 inv = inv_dir(dir);
  const bool exact = !(s.boxes_finite && finite3(org) && finite3(inv));
  hit.t = tfar;
  hit.tri = -1;
  hit.u = hit.v = 0.f;
  int2 stack[kWideStack];
  WideTrav w;
  wide_begin(w, s.wroot);
  if (exact) {
    while (wide_step_rt<true>(s.wnodes, s.wleaves, s.tris, org, inv, dir, hit, w, stack, any)) {
    }
  } else {
    while (wide_step_rt<false>(s.wnodes, s.wleaves, s.tris, org, inv, dir, hit, w, stack, any)) {
    }
  }
  aborted = wide_aborted(w);
  return w.any_hit || hit.tri >= 0;
}

// the 4-wide tree only (kernels specialised for scenes without an 8-wide tree)
template <bool kAny>
DEV bool traverse_wide4(const DevScene& s, v3 org, v3 dir, float tfar, Hit& hit, bool& aborted) {
  v3 inv = inv_dir(dir);
  if (s.boxes_finite && finite3(org) && finite3(inv))
    return traverse_wide_impl<kAny, false>(s, org, inv, dir, tfar, hit, aborted);
  return traverse_wide_impl<kAny, true>(s, org, inv, dir, tfar, hit, aborted);
}

// the scene's wide tree: the compressed 8-wide one where it has one
template <bool kAny>
DEV bool traverse_wide(const DevScene& s, v3 org, v3 dir, float tfar, Hit& hit, bool& aborted) {
  if (s.cnodes) return traverse_cw8_rt(s, org, dir, tfar, kAny, hit, aborted);
  return traverse_wide4<kAny>(s, org, dir, tfar, hit, aborted);
}

template <bool kAny>
DEV bool traverse(const DevScene& s, v3 org, v3 dir, float tfar, Hit& hit, bool& aborted, uint32_t* nodes_visited = nullptr,
                  uint32_t* tris_tested = nullptr) {
  v3 inv = inv_dir(dir);
  if (s.boxes_finite && finite3(org) && finite3(inv))
    return traverse_impl<kAny, false>(s, org, inv, dir, tfar, hit, aborted, nodes_visited, tris_tested);
  return traverse_impl<kAny, true>(s, org, inv, dir, tfar, hit, aborted, nodes_visited, tris_tested);
}

// ---- camera (renderer.frag:129-142, renderer.ts:399-404) -------------------------
struct Camera {
  float m[9];          // mat3(u_u_view_mat), column-major
  float pos[3];
  float film_height;   // u_camera_pos.w = tan(fov/2) * near
  float focal;         // u_focal_length = near
  float inv_res[2];
  int width, height;
};

// v_uv of the pixel centre of the full-screen quad: (2x+1)/W - 1
DEV void camera_ray(const Camera& c, int px, int py, float r0, float r1, v3& org, v3& dir) {
  float vx = __fsub_rn(__fdiv_rn(float(2 * px + 1), float(c.width)), 1.f);
  float vy = __fsub_rn(__fdiv_rn(float(2 * py + 1), float(c.height)), 1.f);
  float ox = __fmul_rn(r0, c.inv_res[0]), oy = __fmul_rn(r1, c.inv_res[1]);
  float aspect = __fdiv_rn(c.inv_res[1], c.inv_res[0]);
  float ux = __fmul_rn(__fadd_rn(__fmul_rn(vx, aspect), ox), c.film_height);
  float uy = __fmul_rn(__fadd_rn(__fmul_rn(vy, 1.f), oy), c.film_height);
  v3 d = normalize_rn(mk(ux, uy, -c.focal));
  v3 c0 = mk(c.m[0], c.m[1], c.m[2]), c1 = mk(c.m[3], c.m[4], c.m[5]), c2 = mk(c.m[6], c.m[7], c.m[8]);
  dir = add_rn(add_rn(mul_rn(c0, d.x), mul_rn(c1, d.y)), mul_rn(c2, d.z));
  org = mk(c.pos[0], c.pos[1], c.pos[2]);
}

// ---- environment (lighting.glsl:24-98, utils.glsl:125-154) ---------------------------
DEV v3 rotate_phi(v3 d, float angle) {
  float s, c;
  sincosf(angle, &s, &c);
  return mk(c * d.x - s * d.z, d.y, s * d.x + c * d.z);
}
DEV float sin_theta_pdf(float theta) { return 1.f / (2.f * kGlslPi * kGlslPi * fmaxf(kEpsCos, sinf(theta))); }
DEV void dir_to_uv(v3 d, float& u, float& v, float& pdf) {
  float theta = acosf(fmaxf(-1.f, fminf(1.f, d.y)));
  float phi = atan2f(d.z, d.x);
  if (phi < 0.f) phi = kGlslTwoPi + phi;
  u = phi / kGlslTwoPi;
  v = theta / kGlslPi;
  pdf = sin_theta_pdf(theta);
}
DEV v3 uv_to_dir(float u, float v, float& pdf) {
  float theta = v * kGlslPi, phi = u * kGlslTwoPi;
  pdf = sin_theta_pdf(theta);
  float st = sinf(theta);
  return mk(st * cosf(phi), cosf(theta), st * sinf(phi));
}
DEV int wrap(int i, int n) {
  int m = i % n;
  return m < 0 ? m + n : m;
}
DEV float4 env_texel(const DevIbl& e, int x, int y) { return __ldg(e.rgba + size_t(y) * e.w + x); }
// texture() with LINEAR filtering and REPEAT wrapping, level 0
DEV v3 env_bilinear(const DevIbl& e, float u, float v) {
  float fu = u * float(e.w) - 0.5f, fv = v * float(e.h) - 0.5f;
  float u0 = floorf(fu), v0 = floorf(fv);
  float a = fu - u0, b = fv - v0;
  int i0 = wrap(int(u0), e.w), j0 = wrap(int(v0), e.h);
  int i1 = wrap(int(u0) + 1, e.w), j1 = wrap(int(v0) + 1, e.h);
  float4 t00 = env_texel(e, i0, j0), t10 = env_texel(e, i1, j0), t01 = env_texel(e, i0, j1), t11 = env_texel(e, i1, j1);
  float w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
  return mk(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x, w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
            w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z);
}
DEV v3 ibl_eval(const DevIbl& e, float rot, v3 d) {
  float u, v, pdf;
  dir_to_uv(rotate_phi(d, rot), u, v, pdf);
  return env_bilinear(e, u, v);
}
// lower_bound over a float CDF (utils.glsl:196-217)
DEV int lower_bound(const float* data, int size, float value) {
  int count = size, first = 0;
  while (count > 0) {
    int step = count / 2;
    int idx = first + step;
    if (__ldg(data + idx) < value) { first = idx + 1; count -= step + 1; }
    else count = step;
  }
  return first;
}
// ibl_sample_direction (lighting.glsl:32-42, 74-84).  mode 1: the reference's
// binary searches; mode 0: the alias table over the same pixel pmf.
DEV v3 ibl_sample(const DevIbl& e, float rot, int mode, float r0, float r1, float& pdf_out) {
  int x, y;
  float pdf_y, pdf_x;
  if (mode == 1) {
    int yi = lower_bound(e.ycdf, e.h, r1);
    pdf_y = yi < e.h ? __ldg(e.ypdf + yi) : 0.f;
    y = yi >= e.h ? e.h - 1 : yi;
    const float* row = e.cdf + size_t(y) * e.w;
    int xi = lower_bound(row, e.w, r0);
    pdf_x = xi < e.w ? __ldg(e.pdf + size_t(y) * e.w + xi) : 0.f;
    x = xi >= e.w ? e.w - 1 : xi;
  } else {
    int n = e.w * e.h;
    int i = min(int(r1 * float(n)), n - 1);
    if (r0 >= __ldg(e.alias_prob + i)) i = __ldg(e.alias_idx + i);
    y = i / e.w;
    x = i - y * e.w;
    pdf_y = __ldg(e.ypdf + y);
    pdf_x = __ldg(e.pdf + i);
  }
  float spdf = float(e.w) * float(e.h) * pdf_y * pdf_x;
  float pdf_w;
  v3 d = uv_to_dir(float(x) / float(e.w), float(y) / float(e.h), pdf_w);
  pdf_out = spdf * pdf_w;
  return rotate_phi(d, -rot);
}
DEV float ibl_pdf(const DevIbl& e, float rot, v3 d) {
  float u, v, pdf_w;
  dir_to_uv(rotate_phi(d, rot), u, v, pdf_w);
  float w = float(e.w), h = float(e.h);
  float x = fminf(u * w, w - 1.f), y = fminf(v * h, h - 1.f);
  int xi = int(x), yi = int(y);
  float py = (yi >= 0 && yi < e.h) ? __ldg(e.ypdf + yi) : 0.f;
  float px = (xi >= 0 && yi >= 0 && xi < e.w && yi < e.h) ? __ldg(e.pdf + size_t(yi) * e.w + xi) : 0.f;
  return w * h * py * px * pdf_w;
}

// ---- hit set-up: fillRenderState + configure_gltf_material -------------------------
struct Surface {
  Closure c;
  v3 n, ng;          // fixed to the incident side (fix_normals, utils.glsl:79-89)
  v3 emissive;
  v3 att_color;
  float att_dist;
  float cutout;
  bool backside, thin_walled;
  v3 pos;
};

DEV float4 vtx(const DevScene& s, uint32_t vi, int slot) { return __ldg(s.verts + 5 * size_t(vi) + slot); }

// get_onb(n) (utils.glsl:97-102): Spencer & Jones basis, first column
DEV v3 onb_tangent(v3 n) { return normalize(cross(n, mk(-n.z, n.x, -n.y))); }

// ---- material textures (the reference's generated texture accessor,
// scene_data_webgl2.ts:318-363) -------------------------------------------------------
// texture(sampler2DArray, vec3) with LINEAR + REPEAT filtering on UNORM8
// texels: the texel coordinates use IEEE-rounded operations so that the
// texels chosen are those of the reference arithmetic.
DEV float4 texel8(const DevTexArray& t, int i, int j, int l) {
  uchar4 c = __ldg(t.data + (size_t(l) * t.h + j) * t.w + i);
  return make_float4(__fdiv_rn(float(c.x), 255.f), __fdiv_rn(float(c.y), 255.f), __fdiv_rn(float(c.z), 255.f),
                     __fdiv_rn(float(c.w), 255.f));
}
DEV int wrap_repeat(int i, int n) {
  int m = i % n;
  return m < 0 ? m + n : m;
}
DEV float4 tex_array_sample(const DevTexArray& t, float u, float v, float layer) {
  float lf = floorf(__fadd_rn(layer, 0.5f));
  int l = lf < 0.f ? 0 : (lf > float(t.layers - 1) ? t.layers - 1 : int(lf));
  float uu = __fsub_rn(__fmul_rn(u, float(t.w)), 0.5f), vv = __fsub_rn(__fmul_rn(v, float(t.h)), 0.5f);
  float fu = floorf(uu), fv = floorf(vv);
  float a = __fsub_rn(uu, fu), b = __fsub_rn(vv, fv);
  int iu = int(fu), iv = int(fv);
  int i0 = wrap_repeat(iu, t.w), j0 = wrap_repeat(iv, t.h), i1 = wrap_repeat(iu + 1, t.w), j1 = wrap_repeat(iv + 1, t.h);
  float4 t00 = texel8(t, i0, j0, l), t10 = texel8(t, i1, j0, l), t01 = texel8(t, i0, j1, l), t11 = texel8(t, i1, j1, l);
  float w00 = __fmul_rn(__fsub_rn(1.f, a), __fsub_rn(1.f, b)), w10 = __fmul_rn(a, __fsub_rn(1.f, b));
  float w01 = __fmul_rn(__fsub_rn(1.f, a), b), w11 = __fmul_rn(a, b);
  auto mix4 = [&](float x00, float x10, float x01, float x11) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(w00, x00), __fmul_rn(w10, x10)), __fmul_rn(w01, x01)),
                     __fmul_rn(w11, x11));
  };
  return make_float4(mix4(t00.x, t10.x, t01.x, t11.x), mix4(t00.y, t10.y, t01.y, t11.y),
                     mix4(t00.z, t10.z, t01.z, t11.z), mix4(t00.w, t10.w, t01.w, t11.w));
}
// get_texture_value(id, uv0, uv1); uv1 is never filled by the reference
// (RenderState.uv1 stays zero).
NOINL float4 texture_value(const DevScene& s, float id, float u0, float v0) {
  const int idx = int(id);
  float4 i0 = make_float4(0.f, 0.f, 0.f, 0.f), i1 = i0;  // a TexInfo beyond the table reads as zeros
  if (idx >= 0 && idx < s.num_texinfo) {
    i0 = __ldg(s.texinfo + 2 * size_t(idx));
    i1 = __ldg(s.texinfo + 2 * size_t(idx) + 1);
  }
  const float u = i1.z > 0.5f ? 0.f : u0, v = i1.z > 0.5f ? 0.f : v0;
  const int arr = int(i0.z);
  if (arr < 0 || arr >= s.num_tex_arrays) return make_float4(1.f, 1.f, 1.f, 1.f);
  return tex_array_sample(s.tex_arrays[arr], __fadd_rn(__fmul_rn(u, i1.x), i0.x), __fadd_rn(__fmul_rn(v, i1.y), i0.y),
                          i0.w);
}
DEV v3 to_linear_rgb(float4 c) { return mk(powf(c.x, 2.2f), powf(c.y, 2.2f), powf(c.z, 2.2f)); }

// configure_gltf_material (material.glsl:5-110) from the interpolated render
// state: material record, textures, vertex colour, normal map, fix_normals,
// anisotropy rotation, closure.  n / ng / tangent as fillRenderState leaves
// them (not yet flipped to the incident side).  kTextured = false is the
// variant for scenes without textures: every texture id reads as unset (-1),
// which is what those scenes' materials hold.
template <bool kTextured>
NOINL Surface configure_gltf(const DevScene& s, int mat, v3 n, v3 ng, float4 tangent, v3 wi, float u0, float v0,
                             float4 vcol, bool lean) {
  Surface S;
  mat = min(max(mat, 0), s.num_materials - 1);
  const float4* m = s.materials + 17 * size_t(mat);
  float4 m0 = __ldg(m + 0), m1 = __ldg(m + 1), m2 = __ldg(m + 2), m3 = __ldg(m + 3), m4 = __ldg(m + 4),
         m5 = __ldg(m + 5), m6 = __ldg(m + 6), m7 = __ldg(m + 7), m8 = __ldg(m + 8), m9 = __ldg(m + 9),
         m10 = __ldg(m + 10), m15 = __ldg(m + 15), m16 = __ldg(m + 16);
  // texture ids (material.ts layout): 39 diffuseTransmission, 44 baseColor,
  // 45 metallicRoughness, 46 normal, 47 emissive, 48 specular, 49 specularColor,
  // 50 transmission, 51 clearcoat, 52 clearcoatRoughness, 54 sheenColor,
  // 55 sheenRoughness, 56 anisotropy, 57 anisotropyDirection, 58 iridescence,
  // 59 iridescenceThickness, 63 diffuseTransmissionColor
  const float4 one = make_float4(1.f, 1.f, 1.f, 1.f);
  float4 m11 = one, m12 = one, m13 = one, m14 = one;
  if (kTextured) {
    m11 = __ldg(m + 11); m12 = __ldg(m + 12); m13 = __ldg(m + 13); m14 = __ldg(m + 14);
  } else {
    m11 = m12 = m13 = m14 = make_float4(-1.f, -1.f, -1.f, -1.f);
    m9.w = -1.f;
    m15.w = -1.f;
  }
  auto tex = [&](float id) { return id < 0.f ? one : texture_value(s, id, u0, v0); };
  GltfMaterial g;
  float4 bc = tex(m11.x);
  g.base_color = m11.x < 0.f ? mk(m0) : mk(m0) * to_linear_rgb(bc);
  float opacity = bc.w;
  if (sqrtf(vcol.x * vcol.x + vcol.y * vcol.y + vcol.z * vcol.z + vcol.w * vcol.w) > 0.f) {
    g.base_color = g.base_color * mk(vcol);
    opacity = opacity * vcol.w;
  }
  float cutout = m2.x * opacity;
  if (m6.w > 0.f) cutout = cutout < m6.w ? 0.f : 1.f;
  if (m6.w == 1.f) cutout = 1.f;
  g.transmission = m12.z < 0.f ? m1.w : m1.w * tex(m12.z).x;
  g.diffuse_transmission = m9.w < 0.f ? m6.z : m6.z * tex(m9.w).x;
  g.diffuse_transmission_color = m15.w < 0.f ? mk(m15) : mk(m15) * to_linear_rgb(tex(m15.w));
  bool thin = m8.w > 0.5f;
  g.ior = m2.w;
  float4 orm = tex(m11.y);
  g.metallic = m11.y < 0.f ? m0.w : m0.w * orm.z;
  g.roughness = m11.y < 0.f ? m1.x : m1.x * orm.y;
  float4 aniso = tex(m14.x);
  g.anisotropy = m14.x < 0.f ? m1.y : m1.y * aniso.z;
  if (m12.y < 0.f) {
    g.specular_color = mk(m3);
  } else {
    float4 sc = tex(m12.y);
    g.specular_color = mk(m3) * mk(powf(sc.x, 2.2f), powf(sc.y, 2.2f), powf(sc.z, 2.2f));
  }
  g.specular = m12.x < 0.f ? m3.w : m3.w * tex(m12.x).w;
  g.sheen_roughness = m13.w < 0.f ? m4.w : m4.w * tex(m13.w).x;
  g.sheen_color = m13.z < 0.f ? mk(m4) : mk(m4) * to_linear_rgb(tex(m13.z));
  v3 t3 = mk(tangent.x, tangent.y, tangent.z);
  if (m11.z >= 0.f) {  // normal map (material.glsl:55-64)
    v3 b = normalize(cross(n, t3));
    v3 tt = cross(b, n);
    float4 tn = tex(m11.z);
    v3 nt = normalize(mk(tn.x, tn.y, tn.z) * 2.0f - mk(1.f));
    nt = normalize(nt * mk(m2.z, m2.z, 1.f));
    n = tt * nt.x + b * nt.y + n * nt.z;
    v3 b2 = normalize(cross(n, t3)) * tangent.w;
    t3 = cross(b2, n);
  }
  // fix_normals (utils.glsl:88-98)
  bool back = false;
  if (dot(wi, ng) < 0.f) { ng = -ng; back = true; }
  if (dot(ng, n) < 0.f) n = -n;
  // anisotropy direction -> rotation -> tangent (material.glsl:71-82, utils.glsl:183-190)
  float ax = m9.x, ay = m9.y;
  if (m14.y >= 0.f) {
    float4 ad = tex(m14.y);
    ax = ad.x * 2.0f - 1.f;
    ay = ad.y * 2.0f - 1.f;
  } else if (m14.x >= 0.f) {
    ax = aniso.x * 2.0f - 1.f;
    ay = aniso.y * 2.0f - 1.f;
  }
  float rot = atan2f(ay, ax) + kGlslPi;
  if (rot > 0.f) {
    v3 b = cross(n, t3) * tangent.w;
    float sr, cr;
    sincosf(rot, &sr, &cr);
    t3 = t3 * cr + b * sr;
  }
  g.clearcoat = m12.w < 0.f ? m6.x : m6.x * tex(m12.w).x;
  g.clearcoat_roughness = m13.x < 0.f ? m6.y : m6.y * tex(m13.x).x;
  g.thickness = thin ? 0.f : 1.f;
  g.iridescence = m14.z < 0.f ? m10.x : m10.x * tex(m14.z).x;
  g.iridescence_ior = m10.y;
  g.iridescence_thickness = mixf(m10.z, m10.w, m14.w < 0.f ? 1.f : tex(m14.w).y);
  g.dispersion = m16.x;
  S.c = build_closure(g, t3, lean);
  S.n = n;
  S.ng = ng;
  S.emissive = m11.w < 0.f ? mk(m5) : mk(m5) * to_linear_rgb(tex(m11.w));
  S.att_color = mk(m7);
  S.att_dist = m7.w;
  S.cutout = cutout;
  S.backside = back;
  S.thin_walled = thin;
  return S;
}

// fillRenderState (renderer.frag:72-91, bvh.glsl:84-134) + configure_gltf.
template <bool kTextured>
NOINL Surface make_surface_t(const DevScene& s, int tri, float bu, float bv, v3 hit_pos, v3 wi, bool lean) {
  uint32_t i0 = __ldg(s.indices + 3 * size_t(tri)), i1 = __ldg(s.indices + 3 * size_t(tri) + 1),
           i2 = __ldg(s.indices + 3 * size_t(tri) + 2);
  float4 q0 = vtx(s, i0, 0), q1 = vtx(s, i1, 0), q2 = vtx(s, i2, 0);
  v3 p0 = mk(q0), p1 = mk(q1), p2 = mk(q2);
  float w0 = 1.f - bu - bv;
  v3 ng = normalize(cross(p1 - p0, p2 - p0));
  v3 n = normalize(w0 * mk(vtx(s, i0, 1)) + bu * mk(vtx(s, i1, 1)) + bv * mk(vtx(s, i2, 1)));
  float4 t0 = vtx(s, i0, 3), t1 = vtx(s, i1, 3), t2 = vtx(s, i2, 3);
  float hand = (t0.w == t1.w && t0.w == t2.w) ? t0.w : 0.f;
  v3 tg = normalize(w0 * mk(t0) + bu * mk(t1) + bv * mk(t2));
  float4 tangent;
  if (length(tg) > 0.99f && fabsf(hand) > 0.99f) tangent = make_float4(tg.x, tg.y, tg.z, -hand);
  else { v3 o = onb_tangent(n); tangent = make_float4(o.x, o.y, o.z, 1.f); }
  float4 c0 = vtx(s, i0, 4), c1 = vtx(s, i1, 4), c2 = vtx(s, i2, 4);
  float4 vcol = make_float4(w0 * c0.x + bu * c1.x + bv * c2.x, w0 * c0.y + bu * c1.y + bv * c2.y,
                            w0 * c0.z + bu * c1.z + bv * c2.z, w0 * c0.w + bu * c1.w + bv * c2.w);
  float u0 = 0.f, v0 = 0.f;
  if (kTextured) {  // compute_interpolated_uv(set 0) (bvh.glsl:108-116)
    float4 a = vtx(s, i0, 2), b = vtx(s, i1, 2), c = vtx(s, i2, 2);
    u0 = w0 * a.x + bu * b.x + bv * c.x;
    v0 = w0 * a.y + bu * b.y + bv * c.y;
  }
  Surface S = configure_gltf<kTextured>(s, int(uint32_t(q0.w)), n, ng, tangent, wi, u0, v0, vcol, lean);
  S.pos = hit_pos;
  return S;
}


}  // namespace dspbr
