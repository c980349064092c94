// Display epilogue: the reference's post-processing passes on the device.
//
// The reference presents a frame by drawing the accumulation texture through
// tonemap.frag into the "postprocess" RGBA32F buffer, optionally through
// fxaa.frag, and then onto the 8-bit canvas (renderer.ts:666-700).  Here the
// tone mapping is fused with the mean of the FP64 pixel sums (one pass over
// the accumulator), FXAA is a gather pass over the tone-mapped image, and the
// 8-bit conversion is fused into whichever pass writes the output.
//
// Arithmetic follows the shaders operation by operation; this file is built
// without FMA contraction (-fmad=false), so every step rounds like the
// shader's.  Textures of the postprocess chain are NEAREST + CLAMP_TO_EDGE
// (gl_utils.ts:22-30), so a texture() lookup is the texel floor(uv * size).
#include <cuda_runtime.h>

#include "display.h"

namespace dspbr {

namespace {

struct f3 {
  float x, y, z;
};
__device__ __forceinline__ f3 mk3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 operator*(f3 a, f3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ f3 operator/(f3 a, f3 b) { return mk3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ f3 operator+(f3 a, float s) { return mk3(a.x + s, a.y + s, a.z + s); }
__device__ __forceinline__ f3 operator-(f3 a, float s) { return mk3(a.x - s, a.y - s, a.z - s); }
// GLSL min / max / clamp (GLSL ES 3.00 8.3): min(x, y) = y < x ? y : x
__device__ __forceinline__ float gmin(float x, float y) { return y < x ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return x < y ? y : x; }
__device__ __forceinline__ float sat(float x) { return gmin(gmax(x, 0.0f), 1.0f); }
__device__ __forceinline__ f3 sat(f3 a) { return mk3(sat(a.x), sat(a.y), sat(a.z)); }
__device__ __forceinline__ f3 vmax(f3 a, float s) { return mk3(gmax(a.x, s), gmax(a.y, s), gmax(a.z, s)); }
__device__ __forceinline__ f3 vmax(float s, f3 a) { return mk3(gmax(s, a.x), gmax(s, a.y), gmax(s, a.z)); }
__device__ __forceinline__ f3 vpow(f3 a, float e) { return mk3(powf(a.x, e), powf(a.y, e), powf(a.z, e)); }
__device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// mat3 (column-major) * vec3: column0 * v.x + column1 * v.y + column2 * v.z
__device__ __forceinline__ f3 mat_mul(const float m[9], f3 v) {
  return mk3(m[0] * v.x, m[1] * v.x, m[2] * v.x) + mk3(m[3] * v.y, m[4] * v.y, m[5] * v.y) +
         mk3(m[6] * v.z, m[7] * v.z, m[8] * v.z);
}

// Uncharted2Helper (tonemap.frag:29-30)
__device__ __forceinline__ f3 uncharted2_helper(f3 x) {
  f3 num = x * (0.15f * x + 0.10f * 0.50f) + 0.20f * 0.02f;
  f3 den = x * (0.15f * x + 0.50f) + 0.20f * 0.30f;
  return vmax((num / den) - 0.02f / 0.30f, 0.0f);
}

// tonemap.frag:72-94 on one colour.  Modes are the renderer's tonemappingModes
// index (renderer.ts:192, 674-675); any other value applies no operator.
__device__ f3 tonemap(f3 color, const DisplayParams& d) {
  const float exposure = d.exposure;
  if (d.mode == 0) {
    color = exposure * color;  // LinearToneMapping
  } else if (d.mode == 1) {  // ReinhardToneMapping
    color = color * exposure;
    color = sat(color / (mk3(1.0f, 1.0f, 1.0f) + color));
  } else if (d.mode == 2) {  // OptimizedCineonToneMapping
    color = color * exposure;
    color = vmax(0.0f, color - 0.004f);
    color = vpow((color * (6.2f * color + 0.5f)) / (color * (6.2f * color + 1.7f) + 0.06f), 2.2f);
  } else if (d.mode == 3) {  // pre-exposure, then ACESFilmicToneMapping
    color = color * (exposure / 0.6f);
    const float in_m[9] = {0.59719f, 0.07600f, 0.02840f, 0.35458f, 0.90834f, 0.13383f, 0.04823f, 0.01566f, 0.83777f};
    const float out_m[9] = {1.60475f, -0.10208f, -0.00327f, -0.53108f, 1.10813f, -0.07276f,
                            -0.07367f, -0.00605f, 1.07602f};
    color = mat_mul(in_m, color);
    f3 a = color * (color + 0.0245786f) - 0.000090537f;  // RRTAndODTFit
    f3 b = color * (0.983729f * color + 0.4329510f) + 0.238081f;
    color = a / b;
    color = mat_mul(out_m, color);
    color = sat(color);
  } else if (d.mode == 4) {  // Uncharted2ToneMapping
    color = color * exposure;
    color = sat(uncharted2_helper(color) / uncharted2_helper(mk3(1.0f, 1.0f, 1.0f)));
  }
  if (d.gamma) color = vpow(color, 1.0f / 2.2f);
  return color;
}

// The canvas conversion of a colour to 8-bit UNORM: clamp to [0, 1], scale by
// 255, round to nearest (GL ES 3.0 2.1.6.2).
__device__ __forceinline__ unsigned char unorm8(float c) { return (unsigned char)__float2uint_rn(sat(c) * 255.0f); }

__device__ __forceinline__ void store(float4* out, size_t i, f3 c, float a) { out[i] = make_float4(c.x, c.y, c.z, a); }
__device__ __forceinline__ void store(uchar4* out, size_t i, f3 c, float a) {
  out[i] = make_uchar4(unorm8(c.x), unorm8(c.y), unorm8(c.z), unorm8(a));
}

// mean of the FP64 sums (the value the reference's running mean holds) ->
// tonemap.frag -> output
template <class Out>
__global__ void k_tonemap(const double4* __restrict__ accum, double inv_count, DisplayParams d, Out* __restrict__ out,
                          int npix) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
    double4 s = accum[i];
    f3 c = mk3(float(s.x * inv_count), float(s.y * inv_count), float(s.z * inv_count));
    float alpha = float(s.w * inv_count);
    store(out, size_t(i), tonemap(c, d), alpha);
  }
}

__device__ __forceinline__ float4 tex_nearest(const float4* __restrict__ img, int w, int h, float u, float v) {
  int i = int(floorf(u * float(w))), j = int(floorf(v * float(h)));
  i = i < 0 ? 0 : (i >= w ? w - 1 : i);
  j = j < 0 ? 0 : (j >= h ? h - 1 : j);
  return __ldg(img + size_t(j) * w + i);
}
__device__ __forceinline__ f3 rgb(float4 t) { return mk3(t.x, t.y, t.z); }

// fxaa.frag:22-64 at fragment (x + 0.5, y + 0.5)
template <class Out>
__global__ void k_fxaa(const float4* __restrict__ img, int w, int h, float inv_w, float inv_h, Out* __restrict__ out) {
  const int npix = w * h;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
    const int x = p % w, y = p / w;
    const float fx = float(x) + 0.5f, fy = float(y) + 0.5f;
    f3 rgbNW = rgb(tex_nearest(img, w, h, (fx + -1.0f) * inv_w, (fy + -1.0f) * inv_h));
    f3 rgbNE = rgb(tex_nearest(img, w, h, (fx + 1.0f) * inv_w, (fy + -1.0f) * inv_h));
    f3 rgbSW = rgb(tex_nearest(img, w, h, (fx + -1.0f) * inv_w, (fy + 1.0f) * inv_h));
    f3 rgbSE = rgb(tex_nearest(img, w, h, (fx + 1.0f) * inv_w, (fy + 1.0f) * inv_h));
    const float cu = fx * inv_w, cv = fy * inv_h;
    float4 texColor = tex_nearest(img, w, h, cu, cv);
    f3 rgbM = rgb(texColor);
    const f3 luma = mk3(0.299f, 0.587f, 0.114f);
    float lumaNW = dot3(rgbNW, luma), lumaNE = dot3(rgbNE, luma), lumaSW = dot3(rgbSW, luma),
          lumaSE = dot3(rgbSE, luma), lumaM = dot3(rgbM, luma);
    float lumaMin = gmin(lumaM, gmin(gmin(lumaNW, lumaNE), gmin(lumaSW, lumaSE)));
    float lumaMax = gmax(lumaM, gmax(gmax(lumaNW, lumaNE), gmax(lumaSW, lumaSE)));
    float dx = -((lumaNW + lumaNE) - (lumaSW + lumaSE));
    float dy = ((lumaNW + lumaSW) - (lumaNE + lumaSE));
    float dirReduce = gmax((lumaNW + lumaNE + lumaSW + lumaSE) * (0.25f * (1.0f / 8.0f)), 1.0f / 128.0f);
    float rcpDirMin = 1.0f / (gmin(fabsf(dx), fabsf(dy)) + dirReduce);
    dx = gmin(8.0f, gmax(-8.0f, dx * rcpDirMin)) * inv_w;
    dy = gmin(8.0f, gmax(-8.0f, dy * rcpDirMin)) * inv_h;
    const float k1 = 1.0f / 3.0f - 0.5f, k2 = 2.0f / 3.0f - 0.5f;
    f3 rgbA = 0.5f * (rgb(tex_nearest(img, w, h, cu + dx * k1, cv + dy * k1)) +
                      rgb(tex_nearest(img, w, h, cu + dx * k2, cv + dy * k2)));
    f3 rgbB = rgbA * 0.5f + 0.25f * (rgb(tex_nearest(img, w, h, cu + dx * -0.5f, cv + dy * -0.5f)) +
                                     rgb(tex_nearest(img, w, h, cu + dx * 0.5f, cv + dy * 0.5f)));
    float lumaB = dot3(rgbB, luma);
    store(out, size_t(p), (lumaB < lumaMin) || (lumaB > lumaMax) ? rgbA : rgbB, texColor.w);
  }
}

// display.frag: the canvas (dw x dh) draws the postprocess buffer (w x h, the
// render resolution) as a full-screen quad; each canvas pixel samples it at
// uv = (x + 0.5) / dw with NEAREST filtering and CLAMP_TO_EDGE
// (gl_utils.ts:22-33, renderer.ts:689-697)
template <class T>
__global__ void k_present(const T* __restrict__ src, int w, int h, T* __restrict__ dst, int dw, int dh) {
  const int n = dw * dh;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int x = p % dw, y = p / dw;
    const float u = (float(x) + 0.5f) / float(dw), v = (float(y) + 0.5f) / float(dh);
    int i = int(floorf(u * float(w))), j = int(floorf(v * float(h)));
    i = i < 0 ? 0 : (i >= w ? w - 1 : i);
    j = j < 0 ? 0 : (j >= h ? h - 1 : j);
    dst[p] = src[size_t(j) * w + i];
  }
}

int grid(int n) {
  int b = (n + 255) / 256;
  return b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b);
}

}  // namespace

void launch_tonemap(const double4* accum, double inv_count, const DisplayParams& d, float4* out, int npix,
                    cudaStream_t st) {
  k_tonemap<float4><<<grid(npix), 256, 0, st>>>(accum, inv_count, d, out, npix);
}
void launch_tonemap8(const double4* accum, double inv_count, const DisplayParams& d, uchar4* out, int npix,
                     cudaStream_t st) {
  k_tonemap<uchar4><<<grid(npix), 256, 0, st>>>(accum, inv_count, d, out, npix);
}
void launch_fxaa(const float4* img, int w, int h, float4* out, cudaStream_t st) {
  k_fxaa<float4><<<grid(w * h), 256, 0, st>>>(img, w, h, 1.0f / float(w), 1.0f / float(h), out);
}
void launch_fxaa8(const float4* img, int w, int h, uchar4* out, cudaStream_t st) {
  k_fxaa<uchar4><<<grid(w * h), 256, 0, st>>>(img, w, h, 1.0f / float(w), 1.0f / float(h), out);
}

void launch_present(const float4* src, int w, int h, float4* dst, int dw, int dh, cudaStream_t st) {
  k_present<float4><<<grid(dw * dh), 256, 0, st>>>(src, w, h, dst, dw, dh);
}
void launch_present8(const uchar4* src, int w, int h, uchar4* dst, int dw, int dh, cudaStream_t st) {
  k_present<uchar4><<<grid(dw * dh), 256, 0, st>>>(src, w, h, dst, dw, dh);
}

}  // namespace dspbr
