// Allocation-free build of the environment-map importance tables.
//
// Some hosts cannot let this library call cudaMalloc: an engine that owns every
// byte of device memory through its own pool and budget, or a real-time frame
// loop where the implicit device synchronisation of cudaMalloc / cudaFree would
// stall the frame.  For them, dspbr_ibl_tables_noalloc builds the same tables
// as dspbr_ibl_create (pdf, cdf, yPdf, yCdf and the total sum, bit for bit)
// into buffers the caller owns, using no allocation at all: its only scratch,
// one float per environment row, lives in the fixed device array below.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library holds its 64 KiB until the process exits.  All calls share it and it
// keeps the contents of the last call; every row sum is rewritten before it is
// read, so nothing needs clearing between calls, but two calls whose kernels
// overlap on the GPU (different streams without ordering) race on it.
//
// The array's device address is looked up once per device and kept.  A host
// that tears the device's context down (cudaDeviceReset) and goes on using the
// device in the same process must not call this entry point afterwards: the
// kept address belongs to the destroyed context.
//
// There is no context object here, so errors are reported on stderr, not
// through dspbr_last_error.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "dspbr.h"

namespace dspbr {
namespace {

constexpr int kNoallocMaxRows = 16384;  // environment maps up to 16384 rows
constexpr int kNoallocMaxDevices = 64;

static __device__ __align__(256) float g_noalloc_rowsum[kNoallocMaxRows];

std::mutex g_setup_mutex;
float* g_rowsum_ptr[kNoallocMaxDevices] = {};

// Luminance of one texel exactly as the table build computes it: double
// arithmetic, rounded to float (renderer.ts:814-820).
__device__ __forceinline__ float texel_luminance(float4 c) {
  double l = __dadd_rn(__dadd_rn(__dmul_rn(double(c.x), 0.299), __dmul_rn(double(c.y), 0.587)),
                       __dmul_rn(double(c.z), 0.114));
  return float(l);
}

// One thread per row: row sum, pdf and cdf with the luminance recomputed from
// the caller's RGBA image instead of a luminance buffer.
__global__ void k_noalloc_rows(const float4* rgba, int w, int h, float* pdf, float* cdf, float* rowsum) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= h) return;
  const float4* row = rgba + size_t(r) * w;
  float* p = pdf + size_t(r) * w;
  float* c = cdf + size_t(r) * w;
  double sum = 0.0;
  for (int i = 0; i < w; ++i) sum = __dadd_rn(sum, double(texel_luminance(row[i])));
  if (sum == 0.0) sum = 1.0;
  for (int i = 0; i < w; ++i) p[i] = float(__ddiv_rn(double(texel_luminance(row[i])), sum));
  c[0] = p[0];
  for (int i = 1; i < w; ++i) c[i] = float(__dadd_rn(double(c[i - 1]), double(p[i])));
  c[w - 1] = 1.0f;
  rowsum[r] = float(sum);
}

// The marginal over the row sums read back from the scratch array.
__global__ void k_noalloc_marginal(const float* rowsum, int h, float* ypdf, float* ycdf, double* total) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double sum = 0.0;
  for (int i = 0; i < h; ++i) sum = __dadd_rn(sum, double(rowsum[i]));
  if (sum == 0.0) sum = 1.0;
  for (int i = 0; i < h; ++i) ypdf[i] = float(__ddiv_rn(double(rowsum[i]), sum));
  ycdf[0] = ypdf[0];
  for (int i = 1; i < h; ++i) ycdf[i] = float(__dadd_rn(double(ycdf[i - 1]), double(ypdf[i])));
  ycdf[h - 1] = 1.0f;
  *total = sum;
}

// Device address of the scratch array on the current device, looked up once
// per device (the first call on a device does this set-up).
int scratch_for_current_device(float** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kNoallocMaxDevices) {
    cudaGetLastError();
    return DSPBR_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_rowsum_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_rowsum);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "dspbr_ibl_tables_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                   cudaGetErrorString(e));
      cudaGetLastError();
      return DSPBR_ERR_CUDA;
    }
    g_rowsum_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_rowsum_ptr[dev];
  return DSPBR_OK;
}

}  // namespace
}  // namespace dspbr

extern "C" int dspbr_ibl_tables_noalloc(const float* rgba32f, int width, int height, float* pdf, float* cdf,
                                        float* ypdf, float* ycdf, double* total_sum, void* stream) {
  using namespace dspbr;
  if (!rgba32f || !pdf || !cdf || !ypdf || !ycdf || !total_sum || width <= 0 || height <= 0)
    return DSPBR_ERR_INVALID;
  // the kernels read the image as float4 and write the total as a double
  if (reinterpret_cast<uintptr_t>(rgba32f) % 16 != 0 || reinterpret_cast<uintptr_t>(total_sum) % 8 != 0 ||
      reinterpret_cast<uintptr_t>(pdf) % 4 != 0 || reinterpret_cast<uintptr_t>(cdf) % 4 != 0 ||
      reinterpret_cast<uintptr_t>(ypdf) % 4 != 0 || reinterpret_cast<uintptr_t>(ycdf) % 4 != 0) {
    std::fprintf(stderr, "dspbr_ibl_tables_noalloc: rgba32f must be 16-byte aligned, total_sum 8-byte aligned and "
                         "the tables 4-byte aligned\n");
    return DSPBR_ERR_INVALID;
  }
  if (height > kNoallocMaxRows) {
    std::fprintf(stderr, "dspbr_ibl_tables_noalloc: environment map has %d rows, this entry point handles at most %d\n",
                 height, kNoallocMaxRows);
    return DSPBR_ERR_INVALID;
  }
  float* rowsum = nullptr;
  int rc = scratch_for_current_device(&rowsum);
  if (rc != DSPBR_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_noalloc_rows<<<(height + 63) / 64, 64, 0, st>>>(reinterpret_cast<const float4*>(rgba32f), width, height, pdf, cdf,
                                                    rowsum);
  k_noalloc_marginal<<<1, 32, 0, st>>>(rowsum, height, ypdf, ycdf, total_sum);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "dspbr_ibl_tables_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return DSPBR_ERR_CUDA;
  }
  return DSPBR_OK;
}
