// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// GLSL ES 3.00 semantics layer used to compile the reference's own fragment
// shader sources (packages/lib/shader/**) as C++ on the host.  The translated
// shader text is produced at build time by glsl2cpp.py into oracle/_ref/ and
// includes this header.  Only tests/, the smoke check and bench.py's CPU
// baseline leg load the resulting library.
//
// Scalar type: GLSL_REAL (float for the FP32 build that performs the shader's
// own arithmetic, double for the FP64 build).  Built-ins follow the GLSL ES
// 3.00 definitions (min/max/clamp/mix/step/reflect/normalize as specified in
// section 8 of the GLSL ES 3.00 spec); transcendental functions use the host
// libm.  Textures follow the WebGL2 sampling rules the reference configures:
// data textures NEAREST/CLAMP via texelFetch (gl_utils.ts:175-201), the
// environment map LINEAR/REPEAT via texture() (gl_utils.ts:203-216).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#undef INFINITY

#ifndef GLSL_REAL
#define GLSL_REAL float
#endif

// Everything lives in namespace glsl so that unqualified calls in the
// translated shader resolve to these GLSL built-ins, not to libm's.
namespace glsl {
typedef GLSL_REAL real;
typedef uint32_t uint;
typedef float f32;  // storage type of the reference's Float32Array / RGBA32F data

static inline real glsl_sqrt(real x) { return std::sqrt(x); }
static inline real sqrt(real x) { return std::sqrt(x); }
static inline real abs(real x) { return std::fabs(x); }
static inline real sin(real x) { return std::sin(x); }
static inline real cos(real x) { return std::cos(x); }
static inline real exp(real x) { return std::exp(x); }
static inline real log(real x) { return std::log(x); }
static inline real acos(real x) { return std::acos(x); }
static inline real atan(real y, real x) { return std::atan2(y, x); }
static inline real pow(real x, real y) { return std::pow(x, y); }
static inline bool isnan(real x) { return std::isnan(x); }
// GLSL ES 3.00 8.3: min(x,y) = y<x ? y : x ; max(x,y) = x<y ? y : x
static inline real min(real x, real y) { return y < x ? y : x; }
static inline real max(real x, real y) { return x < y ? y : x; }
static inline int min(int x, int y) { return y < x ? y : x; }
static inline int max(int x, int y) { return x < y ? y : x; }
static inline real clamp(real x, real a, real b) { return min(max(x, a), b); }
static inline real mix(real x, real y, real a) { return x * (real(1) - a) + y * a; }
static inline real step(real edge, real x) { return x < edge ? real(0) : real(1); }

struct vec2;
struct vec3;
struct vec4;

struct ivec2 {
  int x, y;
  ivec2() : x(0), y(0) {}
  template <class A, class B> ivec2(A a, B b) : x(int(a)), y(int(b)) {}
  explicit ivec2(const vec2& v);
};

struct vec2 {
  union { struct { real x, y; }; struct { real r, g; }; };
  vec2() : x(0), y(0) {}
  explicit vec2(const ivec2& v) : x(real(v.x)), y(real(v.y)) {}
  template <class A> explicit vec2(A a) : x(real(a)), y(real(a)) {}
  template <class A, class B> vec2(A a, B b) : x(real(a)), y(real(b)) {}
  real& operator[](int i) { return i == 0 ? x : y; }
  real operator[](int i) const { return i == 0 ? x : y; }
  vec2 xy() const { return vec2(x, y); }
  vec2 yx() const { return vec2(y, x); }
};

struct vec3 {
  union { struct { real x, y, z; }; struct { real r, g, b; }; };
  vec3() : x(0), y(0), z(0) {}
  template <class A> explicit vec3(A a) : x(real(a)), y(real(a)), z(real(a)) {}
  template <class A, class B, class C> vec3(A a, B b, C c) : x(real(a)), y(real(b)), z(real(c)) {}
  template <class C> vec3(const vec2& v, C c) : x(v.x), y(v.y), z(real(c)) {}
  real& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  real operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  vec2 xy() const { return vec2(x, y); }
  vec2 yx() const { return vec2(y, x); }
  vec2 rg() const { return vec2(x, y); }
  vec3 xyz() const { return *this; }
  vec3 rgb() const { return *this; }
  void set_xyz(const vec3& v) { *this = v; }
};

struct vec4 {
  union { struct { real x, y, z, w; }; struct { real r, g, b, a; }; };
  vec4() : x(0), y(0), z(0), w(0) {}
  template <class A> explicit vec4(A a) : x(real(a)), y(real(a)), z(real(a)), w(real(a)) {}
  template <class A, class B, class C, class D>
  vec4(A a, B b, C c, D d) : x(real(a)), y(real(b)), z(real(c)), w(real(d)) {}
  template <class D> vec4(const vec3& v, D d) : x(v.x), y(v.y), z(v.z), w(real(d)) {}
  real& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  real operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  vec2 xy() const { return vec2(x, y); }
  vec2 yx() const { return vec2(y, x); }
  vec2 zw() const { return vec2(z, w); }
  vec2 rg() const { return vec2(x, y); }
  vec3 xyz() const { return vec3(x, y, z); }
  vec3 rgb() const { return vec3(x, y, z); }
  void set_xyz(const vec3& v) { x = v.x; y = v.y; z = v.z; }
  void set_rgb(const vec3& v) { set_xyz(v); }
  void mul_rgb(const vec3& v) { x *= v.x; y *= v.y; z *= v.z; }
  void mul_xyz(const vec3& v) { mul_rgb(v); }
};

inline ivec2::ivec2(const vec2& v) : x(int(v.x)), y(int(v.y)) {}
struct ivec4 {
  int x, y, z, w;
};
struct uvec2 {
  uint x, y;
  uvec2() : x(0), y(0) {}
  template <class A, class B> uvec2(A a, B b) : x(uint(a)), y(uint(b)) {}
  explicit uvec2(const vec2& v) : x(uint(v.x)), y(uint(v.y)) {}
  uvec2& operator^=(const uvec2& o) { x ^= o.x; y ^= o.y; return *this; }
};

// ---- component-wise arithmetic -------------------------------------------
#define GLSL_VEC_OPS(V, N)                                                              \
  static inline V operator+(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] + b[i]; return r; } \
  static inline V operator-(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] - b[i]; return r; } \
  static inline V operator*(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] * b[i]; return r; } \
  static inline V operator/(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] / b[i]; return r; } \
  static inline V operator+(const V& a, real s) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] + s; return r; }        \
  static inline V operator-(const V& a, real s) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] - s; return r; }        \
  static inline V operator*(const V& a, real s) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] * s; return r; }        \
  static inline V operator/(const V& a, real s) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] / s; return r; }        \
  static inline V operator+(real s, const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = s + a[i]; return r; }        \
  static inline V operator-(real s, const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = s - a[i]; return r; }        \
  static inline V operator*(real s, const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = s * a[i]; return r; }        \
  static inline V operator/(real s, const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = s / a[i]; return r; }        \
  static inline V operator-(const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = -a[i]; return r; }                   \
  static inline V& operator+=(V& a, const V& b) { for (int i = 0; i < N; ++i) a[i] += b[i]; return a; }                \
  static inline V& operator-=(V& a, const V& b) { for (int i = 0; i < N; ++i) a[i] -= b[i]; return a; }                \
  static inline V& operator*=(V& a, const V& b) { for (int i = 0; i < N; ++i) a[i] *= b[i]; return a; }                \
  static inline V& operator/=(V& a, const V& b) { for (int i = 0; i < N; ++i) a[i] /= b[i]; return a; }                \
  static inline V& operator*=(V& a, real s) { for (int i = 0; i < N; ++i) a[i] *= s; return a; }                       \
  static inline V& operator/=(V& a, real s) { for (int i = 0; i < N; ++i) a[i] /= s; return a; }                       \
  static inline V min(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = min(a[i], b[i]); return r; }   \
  static inline V max(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = max(a[i], b[i]); return r; }   \
  static inline V min(const V& a, real b) { V r; for (int i = 0; i < N; ++i) r[i] = min(a[i], b); return r; }          \
  static inline V max(const V& a, real b) { V r; for (int i = 0; i < N; ++i) r[i] = max(a[i], b); return r; }          \
  static inline V clamp(const V& x, const V& a, const V& b) { return min(max(x, a), b); }                               \
  static inline V clamp(const V& x, real a, real b) { V r; for (int i = 0; i < N; ++i) r[i] = clamp(x[i], a, b); return r; } \
  static inline V mix(const V& x, const V& y, const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = mix(x[i], y[i], a[i]); return r; } \
  static inline V mix(const V& x, const V& y, real a) { V r; for (int i = 0; i < N; ++i) r[i] = mix(x[i], y[i], a); return r; } \
  static inline V abs(const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = abs(a[i]); return r; }                    \
  static inline V sqrt(const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = sqrt(a[i]); return r; }                  \
  static inline V exp(const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = exp(a[i]); return r; }                    \
  static inline V log(const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = log(a[i]); return r; }                    \
  static inline V sin(const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = sin(a[i]); return r; }                    \
  static inline V cos(const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = cos(a[i]); return r; }                    \
  static inline V pow(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = pow(a[i], b[i]); return r; }  \
  static inline real dot(const V& a, const V& b) { real s = a[0] * b[0]; for (int i = 1; i < N; ++i) s = s + a[i] * b[i]; return s; } \
  static inline real length(const V& a) { return sqrt(dot(a, a)); }                                                    \
  static inline V normalize(const V& a) { return a / length(a); }

GLSL_VEC_OPS(vec2, 2)
GLSL_VEC_OPS(vec3, 3)
GLSL_VEC_OPS(vec4, 4)

static inline vec3 cross(const vec3& a, const vec3& b) {
  return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static inline vec3 reflect(const vec3& I, const vec3& N) { return I - real(2) * dot(N, I) * N; }

// Column-major matrices (GLSL convention).
struct mat3 {
  vec3 c[3];
  mat3() {}
  mat3(const vec3& a, const vec3& b, const vec3& d) { c[0] = a; c[1] = b; c[2] = d; }
  template <class T0, class T1, class T2, class T3, class T4, class T5, class T6, class T7, class T8>
  mat3(T0 a0, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7, T8 a8) {
    c[0] = vec3(a0, a1, a2); c[1] = vec3(a3, a4, a5); c[2] = vec3(a6, a7, a8);
  }
  explicit mat3(const struct mat4& m);
  vec3& operator[](int i) { return c[i]; }
  const vec3& operator[](int i) const { return c[i]; }
};
struct mat4 {
  vec4 c[4];
  vec4& operator[](int i) { return c[i]; }
  const vec4& operator[](int i) const { return c[i]; }
};
inline mat3::mat3(const mat4& m) {
  for (int i = 0; i < 3; ++i) c[i] = vec3(m.c[i].x, m.c[i].y, m.c[i].z);
}
static inline vec3 operator*(const mat3& m, const vec3& v) {
  return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z;
}

// ---- textures -------------------------------------------------------------
// texels: 4 (RGBA32F) or 1 (R32F) floats per texel, row-major, row 0 first.
struct sampler2D {
  const float* data = nullptr;
  int w = 0, h = 0, channels = 4;
  bool nearest_clamp = false;  // NEAREST + CLAMP_TO_EDGE (render buffers, gl_utils.ts:22-30)
};
struct isampler2D {
  const int32_t* data = nullptr;
  int w = 0, h = 0;
};
static inline vec4 texelFetch(const sampler2D& s, ivec2 p, int) {
  if (!s.data || p.x < 0 || p.y < 0 || p.x >= s.w || p.y >= s.h) return vec4(0, 0, 0, 0);
  const float* t = s.data + (size_t(p.y) * s.w + p.x) * s.channels;
  if (s.channels == 1) return vec4(t[0], 0, 0, 1);
  return vec4(t[0], t[1], t[2], t[3]);
}
static inline ivec4 texelFetch(const isampler2D& s, ivec2 p, int) {
  if (!s.data || p.x < 0 || p.y < 0 || p.x >= s.w || p.y >= s.h) return ivec4{0, 0, 0, 0};
  return ivec4{s.data[size_t(p.y) * s.w + p.x], 0, 0, 1};
}
static inline int glsl_wrap_repeat(int i, int n) { int m = i % n; return m < 0 ? m + n : m; }
// LINEAR + REPEAT filtering, level 0 (GLSL ES 3.00 / GL ES 3.0 spec 3.8.10),
// or NEAREST + CLAMP_TO_EDGE: texel floor(uv * size) clamped to the image.
static inline vec4 texture(const sampler2D& s, vec2 uv) {
  if (s.nearest_clamp) {
    int i = int(std::floor(uv.x * real(s.w))), j = int(std::floor(uv.y * real(s.h)));
    i = i < 0 ? 0 : (i >= s.w ? s.w - 1 : i);
    j = j < 0 ? 0 : (j >= s.h ? s.h - 1 : j);
    return texelFetch(s, ivec2(i, j), 0);
  }
  real u = uv.x * real(s.w) - real(0.5), v = uv.y * real(s.h) - real(0.5);
  real fu = std::floor(u), fv = std::floor(v);
  real a = u - fu, b = v - fv;
  int i0 = glsl_wrap_repeat(int(fu), s.w), j0 = glsl_wrap_repeat(int(fv), s.h);
  int i1 = glsl_wrap_repeat(int(fu) + 1, s.w), j1 = glsl_wrap_repeat(int(fv) + 1, s.h);
  vec4 t00 = texelFetch(s, ivec2(i0, j0), 0), t10 = texelFetch(s, ivec2(i1, j0), 0);
  vec4 t01 = texelFetch(s, ivec2(i0, j1), 0), t11 = texelFetch(s, ivec2(i1, j1), 0);
  return (real(1) - a) * (real(1) - b) * t00 + a * (real(1) - b) * t10 + (real(1) - a) * b * t01 + a * b * t11;
}

// sampler2DArray of RGBA8 layers (material texture arrays,
// scene_data_webgl2.ts:266-300): UNORM texels c / 255, LINEAR + REPEAT within
// the layer round(layer) clamped to the array (GLSL ES 3.00 8.9, GL ES 3.0 3.8.10).
struct sampler2DArray {
  const uint8_t* data = nullptr;  // layers x h x w x 4
  int w = 0, h = 0, layers = 0;
};
static inline vec4 glsl_texel8(const sampler2DArray& s, int i, int j, int l) {
  const uint8_t* t = s.data + ((size_t(l) * s.h + j) * s.w + i) * 4;
  return vec4(real(t[0]) / real(255), real(t[1]) / real(255), real(t[2]) / real(255), real(t[3]) / real(255));
}
static inline vec4 texture(const sampler2DArray& s, vec3 uvl) {
  if (!s.data || s.layers <= 0) return vec4(0, 0, 0, 0);
  real lf = std::floor(uvl.z + real(0.5));
  int l = lf < real(0) ? 0 : (lf > real(s.layers - 1) ? s.layers - 1 : int(lf));
  real u = uvl.x * real(s.w) - real(0.5), v = uvl.y * real(s.h) - real(0.5);
  real fu = std::floor(u), fv = std::floor(v);
  real a = u - fu, b = v - fv;
  int i0 = glsl_wrap_repeat(int(fu), s.w), j0 = glsl_wrap_repeat(int(fv), s.h);
  int i1 = glsl_wrap_repeat(int(fu) + 1, s.w), j1 = glsl_wrap_repeat(int(fv) + 1, s.h);
  vec4 t00 = glsl_texel8(s, i0, j0, l), t10 = glsl_texel8(s, i1, j0, l);
  vec4 t01 = glsl_texel8(s, i0, j1, l), t11 = glsl_texel8(s, i1, j1, l);
  return (real(1) - a) * (real(1) - b) * t00 + a * (real(1) - b) * t10 + (real(1) - a) * b * t01 + a * b * t11;
}

// Fragment-stage built-ins (per host thread).
extern thread_local vec4 gl_FragCoord;
extern thread_local vec2 v_uv;
extern thread_local vec4 out_FragColor;

}  // namespace glsl
