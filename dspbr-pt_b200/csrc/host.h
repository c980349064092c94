// Host-side helpers shared by the C ABI, the render engine and the server.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "dspbr.h"

namespace dspbr {

// Owning device allocation (cudaMalloc / cudaFree).
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    reset();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e == cudaSuccess) n = count;
    else p = nullptr;
    return e;
  }
  size_t bytes() const { return n * sizeof(T); }
  void swap(DevBuf& o) {
    T* tp = p; p = o.p; o.p = tp;
    size_t tn = n; n = o.n; o.n = tn;
  }
};

// Error reporting into a context's last-error string.
struct Status {
  std::string* err;
  int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (err) *err = buf;
    return code;
  }
  int cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return DSPBR_OK;
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? DSPBR_ERR_OOM : DSPBR_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
  }
};

#define TRY_CUDA(st, expr, what)         \
  do {                                   \
    int rc_ = (st).cuda((expr), (what)); \
    if (rc_ != DSPBR_OK) return rc_;     \
  } while (0)

inline double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace dspbr
