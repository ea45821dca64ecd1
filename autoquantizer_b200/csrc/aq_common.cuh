// Shared host/device helpers of libaq.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/aq.h"

#define AQ_CUDA_TRY(expr)                        \
  do {                                           \
    cudaError_t aq_err_ = (expr);                \
    if (aq_err_ != cudaSuccess) {                \
      aq::set_last_cuda_error(aq_err_, #expr);   \
      return AQ_E_CUDA;                          \
    }                                            \
  } while (0)

namespace aq {

void set_last_cuda_error(cudaError_t e, const char* what);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline int num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

inline unsigned grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 0x7fffffffLL) b = 0x7fffffffLL;
  return (unsigned)b;
}

}  // namespace aq
