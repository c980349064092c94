// Environment-map importance tables on the device.
//
// Reproduces precomputeIBLImportanceSamplingData / precompute1DPdfAndCdf
// (packages/lib/renderer.ts:777-838) bit for bit.  The reference runs in
// JavaScript: luminance, row sums, quotients and prefix steps are evaluated in
// double precision and every stored value is rounded to a Float32Array entry.
// Here the same FP64 arithmetic runs on the GPU: luminance per texel in
// parallel; each row's sum and prefix are accumulated in FP64 in the
// reference's sequential order (one thread per row, rows in parallel) so the
// float32 tables are identical; the marginal over the row sums is one more
// such row.  No FMA contraction is allowed in these steps.
#include <cuda_runtime.h>

#include "kernels.h"

namespace dspbr {

__global__ void k_luminance(const float4* rgba, size_t n, float* lum) {
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
    float4 c = rgba[k];
    double l = __dadd_rn(__dadd_rn(__dmul_rn(double(c.x), 0.299), __dmul_rn(double(c.y), 0.587)),
                         __dmul_rn(double(c.z), 0.114));
    lum[k] = float(l);
  }
}

// precompute1DPdfAndCdf for `rows` rows of length `num`: row sum (FP64,
// left to right), pdf = v / sum, cdf prefix with float32 storage, last = 1.
__global__ void k_pdf_cdf_rows(const float* data, int rows, int num, float* pdf, float* cdf, float* rowsum,
                               double* total) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const float* d = data + size_t(r) * num;
  float* p = pdf + size_t(r) * num;
  float* c = cdf + size_t(r) * num;
  double sum = 0.0;
  for (int i = 0; i < num; ++i) sum = __dadd_rn(sum, double(d[i]));
  if (sum == 0.0) sum = 1.0;
  for (int i = 0; i < num; ++i) p[i] = float(__ddiv_rn(double(d[i]), sum));
  c[0] = p[0];
  for (int i = 1; i < num; ++i) c[i] = float(__dadd_rn(double(c[i - 1]), double(p[i])));
  c[num - 1] = 1.0f;
  if (rowsum) rowsum[r] = float(sum);
  if (total) *total = sum;
}

void launch_ibl_tables(const float4* rgba, int w, int h, float* lum, float* pdf, float* cdf, float* rowsum,
                       float* ypdf, float* ycdf, double* total, cudaStream_t st) {
  size_t n = size_t(w) * h;
  k_luminance<<<148 * 8, 256, 0, st>>>(rgba, n, lum);
  k_pdf_cdf_rows<<<(h + 63) / 64, 64, 0, st>>>(lum, h, w, pdf, cdf, rowsum, nullptr);
  k_pdf_cdf_rows<<<1, 32, 0, st>>>(rowsum, 1, h, ypdf, ycdf, nullptr, total);
}

}  // namespace dspbr
