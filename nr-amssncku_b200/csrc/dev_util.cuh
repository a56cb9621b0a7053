// dev_util.cuh -- host-side error handling and small helpers of the library.
#pragma once
#include <cstdio>
#include <cuda_runtime.h>

#include "amss_b200.h"

namespace amss {

// Records the message for amss_last_error() and echoes it on stderr.
int amss_fail(int code, const char* msg);

// 0 when a CUDA device is usable; otherwise records why and returns -1.
// The library has no CPU path: callers return AMSS_ERR_NO_DEVICE.
int check_device(const char* who);

// Field stride: round a field's point count up to 64 elements so every field
// starts on a 256-byte boundary (FP64) / 128-byte boundary (FP32).
inline long long pad_stride(long long n) { return (n + 63) / 64 * 64; }

}  // namespace amss

#define AMSS_CK(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      char m_[256];                                                                        \
      std::snprintf(m_, sizeof m_, "%s:%d: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
      return ::amss::amss_fail(AMSS_ERR_CUDA, m_);                                         \
    }                                                                                      \
  } while (0)

#define AMSS_CKV(call)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      char m_[256];                                                                        \
      std::snprintf(m_, sizeof m_, "%s:%d: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
      ::amss::amss_fail(AMSS_ERR_CUDA, m_);                                                \
      return;                                                                              \
    }                                                                                      \
  } while (0)
