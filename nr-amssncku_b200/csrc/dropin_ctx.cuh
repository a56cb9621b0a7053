// dropin_ctx.cuh -- per-thread device scratch of the drop-in entry points.
#pragma once
#include <cuda_runtime.h>

#include "dev_util.cuh"

namespace amss {

// Per-thread device scratch of the drop-in entries (grow-only, reused).
struct DropinCtx {
  cudaStream_t stream = nullptr;
  double* dbuf = nullptr;
  size_t cap = 0;      // doubles
  unsigned* dstatus = nullptr;
  bool ok = false;
  ~DropinCtx() {
    if (dbuf) cudaFree(dbuf);
    if (dstatus) cudaFree(dstatus);
    if (stream) cudaStreamDestroy(stream);
  }
  int init() {
    if (ok) return 0;
    if (check_device("drop-in") != 0) return -1;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return -1;
    if (cudaMalloc(&dstatus, sizeof(unsigned)) != cudaSuccess) return -1;
    ok = true;
    return 0;
  }
  double* reserve(size_t n) {
    if (n > cap) {
      if (dbuf) cudaFree(dbuf);
      dbuf = nullptr;
      cap = 0;
      if (cudaMalloc(&dbuf, n * sizeof(double)) != cudaSuccess) return nullptr;
      cap = n;
    }
    return dbuf;
  }
};

// The calling thread's context (one stream and one grow-only buffer per thread).
DropinCtx& dropin_ctx();

}  // namespace amss
