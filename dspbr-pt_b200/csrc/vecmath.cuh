// Small float3 vector layer for the device code.
//
// Two flavours of arithmetic are used on purpose:
//  * default operators allow the compiler to contract into FMA (shading math,
//    compared to the oracle within a stated tolerance);
//  * the *_rn helpers round every operation separately (no contraction), used
//    where results must be bit-identical to IEEE single-precision host code:
//    camera rays, ray/box slabs and Moller-Trumbore (closest-hit triangle ids).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define DEV __device__ __forceinline__
// Large, multiply-called device functions stay out of line: one copy of the
// code keeps the instruction cache of divergent shading warps from thrashing.
#define NOINL static __device__ __noinline__
#define HD __host__ __device__ __forceinline__

namespace dspbr {

struct v3 {
  float x, y, z;
};

DEV v3 mk(float x, float y, float z) { return v3{x, y, z}; }
DEV v3 mk(float s) { return v3{s, s, s}; }
DEV v3 mk(float4 a) { return v3{a.x, a.y, a.z}; }
DEV v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
DEV v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
DEV v3 operator*(v3 a, v3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
DEV v3 operator/(v3 a, v3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
DEV v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
DEV v3 operator*(float s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
DEV v3 operator/(v3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
DEV v3 operator+(v3 a, float s) { return {a.x + s, a.y + s, a.z + s}; }
DEV v3 operator+(float s, v3 a) { return {s + a.x, s + a.y, s + a.z}; }
DEV v3 operator-(v3 a, float s) { return {a.x - s, a.y - s, a.z - s}; }
DEV v3 operator-(float s, v3 a) { return {s - a.x, s - a.y, s - a.z}; }
DEV v3 operator-(v3 a) { return {-a.x, -a.y, -a.z}; }
DEV v3& operator+=(v3& a, v3 b) { a = a + b; return a; }
DEV v3& operator*=(v3& a, v3 b) { a = a * b; return a; }
DEV v3& operator*=(v3& a, float s) { a = a * s; return a; }

// GLSL ES 3.00 min/max/clamp (min(x,y) = y<x ? y : x), identical for NaN-free
// inputs to fminf/fmaxf; the GLSL form is kept where NaN handling matters.
DEV float gmin(float x, float y) { return y < x ? y : x; }
DEV float gmax(float x, float y) { return x < y ? y : x; }
DEV float clampf(float x, float a, float b) { return fminf(fmaxf(x, a), b); }
DEV float sat(float x) { return clampf(x, 0.f, 1.f); }
DEV float mixf(float x, float y, float a) { return x * (1.f - a) + y * a; }
DEV v3 vmax(v3 a, v3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
DEV v3 vmax(v3 a, float s) { return {fmaxf(a.x, s), fmaxf(a.y, s), fmaxf(a.z, s)}; }
DEV v3 vmin(v3 a, v3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
DEV v3 vclamp(v3 a, float lo, float hi) { return {clampf(a.x, lo, hi), clampf(a.y, lo, hi), clampf(a.z, lo, hi)}; }
DEV v3 sat(v3 a) { return vclamp(a, 0.f, 1.f); }
DEV v3 vmix(v3 x, v3 y, float a) { return x * (1.f - a) + y * a; }
DEV float max3(v3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
DEV float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DEV v3 cross(v3 a, v3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
DEV float length(v3 a) { return sqrtf(dot(a, a)); }
DEV v3 normalize(v3 a) { return a * rsqrtf(dot(a, a)); }
DEV v3 reflect(v3 i, v3 n) { return i - 2.f * dot(n, i) * n; }
DEV v3 vexp(v3 a) { return {expf(a.x), expf(a.y), expf(a.z)}; }
DEV v3 vlog(v3 a) { return {logf(a.x), logf(a.y), logf(a.z)}; }
DEV v3 vsqrt(v3 a) { return {sqrtf(a.x), sqrtf(a.y), sqrtf(a.z)}; }
DEV v3 vcos(v3 a) { return {cosf(a.x), cosf(a.y), cosf(a.z)}; }
DEV float pow5(float x) { float x2 = x * x; return x2 * x2 * x; }

// ---- separately rounded arithmetic (bit-exact with IEEE host code) --------
DEV float mul_rn(float a, float b) { return __fmul_rn(a, b); }
DEV float add_rn(float a, float b) { return __fadd_rn(a, b); }
DEV float sub_rn(float a, float b) { return __fsub_rn(a, b); }
DEV v3 sub_rn(v3 a, v3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
DEV v3 mul_rn(v3 a, v3 b) { return {__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z)}; }
DEV v3 mul_rn(v3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
DEV v3 add_rn(v3 a, v3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
DEV float dot_rn(v3 a, v3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
DEV v3 cross_rn(v3 a, v3 b) {
  return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(b.y, a.z)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(b.z, a.x)),
          __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(b.x, a.y))};
}
DEV v3 normalize_rn(v3 a) {
  float l = __fsqrt_rn(dot_rn(a, a));
  return {__fdiv_rn(a.x, l), __fdiv_rn(a.y, l), __fdiv_rn(a.z, l)};
}

}  // namespace dspbr
