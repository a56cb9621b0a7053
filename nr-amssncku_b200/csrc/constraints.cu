// constraints.cu -- the constraint monitor of the engine: L2 norms of the
// 7 constraint residuals of a level's current state (Parallel::L2Norm,
// Parallel.C:4214-4243, with l2normhelper, fmisc.f90:1263-1309).
//
// The residuals are compute_rhs_bssn's with co = 0 (bssn_rhs.f90:1044-1135:
// the Hamiltonian constraint, the 3 momentum constraints, the 3 Gamma
// constraints), always in FP64 from the FP64 state, whatever the engine's
// precision.  A Z4c state adds the L2 norm of Theta (Z4c_class.C:2491-2510:
// compute_rhs_Z4c's residuals are constraint_bssn's, Z4c_rhs.f90:1266-1292,
// the same formulas).  Each block contributes the cells of its region (one
// int[6] of local [lo, hi) per block), weighted by its cell volume.
#include <cuda_runtime.h>

#include "substep_common.cuh"

namespace amss {

struct EpiNone {   // the right-hand side itself is not wanted
  template <int F>
  __device__ __forceinline__ void put(double) {}
  __device__ __forceinline__ void finish() {}
};

constexpr int kConsThreads = 128;

// residuals of every point of the level into cons (7 fields, the D layout:
// block offset doff, field stride dfs)
template <typename T, bool SYMM>
__global__ void __launch_bounds__(kConsThreads) k_constraints(const StepBlock<T>* __restrict__ blocks,
                                                              const int2* __restrict__ tiles, int ntiles, int tile_pts,
                                                              double* __restrict__ cons, long long dfs) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
  for (int e = threadIdx.x; e < tile_pts; e += blockDim.x) {
    const int2 tile = tiles[t];
    const StepBlock<T>& B = blocks[tile.x];
    const long long p = (long long)tile.y + e;
    if (p >= B.npts) continue;
    const double* u = B.tl[B.lvl[0]];
    auto q = make_pt<double, SYMM>(u, B.b, p);
    const PointGates G = point_gates(B.b, q.i, q.j, q.k);
    const Coefs<double> C{B.C.d, B.C.d};
    RhsAux aux{nullptr, nullptr, cons + B.doff, nullptr, dfs, 0};
    EpiNone epi;
    (void)bssn_rhs_point<double, double, SYMM, true>(q, C, G, aux, epi);
  }
}

constexpr int kNorms = 8;   // the 7 residuals, then Theta (Z4c; 0 for BSSN)

// per CTA: sum over the region cells of c^2 dV for the 7 residuals and Theta
template <typename T>
__global__ void __launch_bounds__(kConsThreads) k_constraint_sums(const StepBlock<T>* __restrict__ blocks,
                                                                  const int2* __restrict__ tiles, int ntiles,
                                                                  int tile_pts, const int* __restrict__ region,
                                                                  const double* __restrict__ cons, long long dfs,
                                                                  double* __restrict__ part) {
  double acc[kNorms] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
  for (int e = threadIdx.x; e < tile_pts; e += blockDim.x) {
    const int2 tile = tiles[t];
    const StepBlock<T>& B = blocks[tile.x];
    const long long p = (long long)tile.y + e;
    if (p >= B.npts) continue;
    int i, j, k;
    point_ijk(p, B.b.ex, i, j, k);
    const int* r = region + 6 * tile.x;
    if (i < r[0] || j < r[1] || k < r[2] || i >= r[3] || j >= r[4] || k >= r[5]) continue;
    const double dV = B.b.dx[0] * B.b.dx[1] * B.b.dx[2];
#pragma unroll
    for (int c = 0; c < 7; ++c) {
      const double v = cons[c * dfs + B.doff + p];
      acc[c] += v * v * dV;
    }
    if (B.nf == NFIELDS_Z4C) {
      const double th = B.tl[B.lvl[0]][(long long)F_TZ * B.b.fs + p];
      acc[7] += th * th * dV;
    }
  }
  __shared__ double red[kConsThreads / 32][kNorms];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < kNorms; ++c) {
    double v = acc[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNorms) {
    double v = 0.0;
    for (int w = 0; w < kConsThreads / 32; ++w) v += red[w][threadIdx.x];
    part[blockIdx.x * kNorms + threadIdx.x] = v;
  }
}

// tiles: the level's pointwise tiles (tile_pts points each); part: grid x 8
template <typename T>
cudaError_t launch_constraints(const void* table, const int2* tiles, int ntiles, int tile_pts, bool symm,
                               const int* region, double* cons, long long dfs, double* part, int grid,
                               cudaStream_t s) {
  const StepBlock<T>* bl = (const StepBlock<T>*)table;
  const int g1 = ntiles < 148 * 8 ? ntiles : 148 * 8;
  if (symm)
    k_constraints<T, true><<<g1, kConsThreads, 0, s>>>(bl, tiles, ntiles, tile_pts, cons, dfs);
  else
    k_constraints<T, false><<<g1, kConsThreads, 0, s>>>(bl, tiles, ntiles, tile_pts, cons, dfs);
  k_constraint_sums<T><<<grid, kConsThreads, 0, s>>>(bl, tiles, ntiles, tile_pts, region, cons, dfs, part);
  return cudaGetLastError();
}

template cudaError_t launch_constraints<double>(const void*, const int2*, int, int, bool, const int*, double*,
                                                long long, double*, int, cudaStream_t);
template cudaError_t launch_constraints<float>(const void*, const int2*, int, int, bool, const int*, double*,
                                               long long, double*, int, cudaStream_t);

}  // namespace amss
