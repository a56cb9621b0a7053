// amr_types.cuh -- host/device descriptors of the AMR data movement (amr.cuh).
#pragma once
#include "bssn_step.cuh"

namespace amss {

// Per-block buffers as the AMR kernels see them (one table for all levels).
struct AmrBlock {
  int org[3];          // global level index of array element 0
  int ex[3];
  long long fs;
  double* tl[3];       // three time levels of the FP64 state; tl[cur] is current
  void* st[2];         // stage buffers (FP64, or FP32 in the mixed form)
  double* side[2];     // FP64 chi, alpha, beta^i of the stages (mixed form, kSideFields each)
  double* K;           // RK accumulator, reused as the time-interpolated parent state
  const int* lvl;      // level state {cur, steps taken}
  int nf;              // evolved fields: 24 (BSSN) or 25 (Z4c)
};

// A box of work: [lo, lo + n) in global level indices of the destination.
struct AmrBox {
  int dst, src;        // block ids
  int lo[3];
  int n[3];
};

// Fine cells per thread of the prolongation (a run along x from an even
// index), and the runs that cover x cells [lo0, lo0 + n0) of a box.
constexpr int kProlongRun = 16;
__host__ __device__ inline int prolong_runs_x(int lo0, int n0) {
  return ((lo0 + n0) - (lo0 & ~1) + kProlongRun - 1) / kProlongRun;
}

enum AmrBuf : int { BUF_STATE = 0, BUF_STAGE_A = 1, BUF_STAGE_B = 2, BUF_TEMP = 3 };

}  // namespace amss
