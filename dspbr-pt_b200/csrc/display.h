// Display epilogue kernels (display.cu): tonemap.frag + gamma, fxaa.frag,
// 8-bit canvas conversion.
#pragma once
#include <cuda_runtime.h>

namespace dspbr {

struct DisplayParams {
  float exposure;
  int mode;   // tonemappingModes index (renderer.ts:192); other values: no operator
  int gamma;  // pow(c, 1/2.2)
};

void launch_tonemap(const double4* accum, double inv_count, const DisplayParams& d, float4* out, int npix,
                    cudaStream_t st);
void launch_tonemap8(const double4* accum, double inv_count, const DisplayParams& d, uchar4* out, int npix,
                     cudaStream_t st);
void launch_fxaa(const float4* img, int w, int h, float4* out, cudaStream_t st);
void launch_fxaa8(const float4* img, int w, int h, uchar4* out, cudaStream_t st);
// display.frag: nearest-neighbour resampling of the w x h postprocess buffer
// onto the dw x dh canvas
void launch_present(const float4* src, int w, int h, float4* dst, int dw, int dh, cudaStream_t st);
void launch_present8(const uchar4* src, int w, int h, uchar4* dst, int dw, int dh, cudaStream_t st);

}  // namespace dspbr
