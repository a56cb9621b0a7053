// substep_impl.cuh -- the fused RK4 substep kernel template and its launcher.
// Instantiated in one translation unit per (precision, symmetry) pair so the
// large kernels compile in parallel.
#pragma once
#include "substep_common.cuh"

#ifndef AMSS_SUBSTEP_MINB   // resident CTAs of 128 threads the register-pass kernel is compiled for
#define AMSS_SUBSTEP_MINB 2
#endif
#ifndef AMSS_SUBSTEP_MINB_F32   // the same for FP32 arithmetic (fits 168 registers without spills)
#define AMSS_SUBSTEP_MINB_F32 3
#endif
#ifndef AMSS_POINTWISE_PREFETCH   // L2 prefetch in the register pass: 0 none, 1 the next tile's rows, 2 this
#define AMSS_POINTWISE_PREFETCH 2     // tile's, 3 both
#endif

namespace amss {

// Region of a tile: -1 the whole array, else the index into StepBlock::rlo/rn.
__device__ __forceinline__ int tile_region(int x) {
  return (x & kRegionTile) ? ((x & kOwnRegion) ? 1 : 0) : -1;
}

// Points of a tile list's range in a block: its array, or one of its regions.
template <typename T>
__device__ __forceinline__ long long tile_count(const StepBlock<T>& B, int rg) {
  return rg >= 0 ? (long long)B.rn[rg][0] * B.rn[rg][1] * B.rn[rg][2] : B.npts;
}

// Array point of entry q of a tile's point range, or -1 past its end.
template <typename T>
__device__ __forceinline__ long long tile_point(const StepBlock<T>& B, int rg, long long q) {
  if (q >= tile_count(B, rg)) return -1;
  if (rg < 0) return q;
  const int* lo = B.rlo[rg];
  const int* n = B.rn[rg];
  const long long n01 = (long long)n[0] * n[1];
  const int k = (int)(q / n01);
  const long long r = q - (long long)k * n01;
  const int j = (int)(r / n[0]), i = (int)(r - (long long)j * n[0]);
  return (long long)(i + lo[0]) + (long long)B.b.ex[0] * ((long long)(j + lo[1]) + (long long)B.b.ex[1] * (k + lo[2]));
}

// Fused RK4 substep over a tile list of one level.  Substep `sub` reads
// (sub0: u0, sub1: A, sub2: B, sub3: A) and writes (A, B, A, unew).
// SPLIT: the stencil terms come from the D array the stencil pass (k_deriv)
// wrote for this substep; otherwise every stencil is evaluated here.
template <typename T, typename SI, typename SO, bool SYMM, bool SPLIT, bool Z4C>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? AMSS_SUBSTEP_MINB_F32 : AMSS_SUBSTEP_MINB) k_substep(const StepBlock<T>* __restrict__ blocks,
                                                                    const int2* __restrict__ tiles, int ntiles,
                                                                    int sub, RKConst rk, int enforce,
                                                                    unsigned* status, const T* __restrict__ D,
                                                                    long long dfs) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 tile = tiles[t];
    const int region = tile_region(tile.x);
    const StepBlock<T>& B = blocks[tile.x & kTileIndex];
#if AMSS_POINTWISE_PREFETCH
    // split form: pull the rows of a tile (D slots, stage input, u0, K) into
    // L2 -- the next tile's while this one computes, or this tile's before its
    // point function issues its loads one by one -- so they meet L2 rather
    // than HBM latency
    if constexpr (SPLIT) {
#pragma unroll 1
     for (int pass = 0; pass < 2; ++pass) {
      const int mode = AMSS_POINTWISE_PREFETCH;
      if (pass == 0 ? !(mode & 2) : !(mode & 1)) continue;
      const int tn = pass == 0 ? t : t + (int)gridDim.x;
      if (threadIdx.x < 32 && tn < ntiles) {
        const int2 nt = tiles[tn];
        const int nreg = tile_region(nt.x);
        const StepBlock<T>& N = blocks[nt.x & kTileIndex];
        const long long fs = N.b.fs;
        const int cur = N.lvl[0];
        const SI* nin = sub == 0 ? (const SI*)N.tl[cur] : (const SI*)N.stage[sub == 2 ? 1 : 0];
        // the array span of the tile's points (the last tile of a block is short; a
        // region tile's rows are strided, the span holds them), at most two tiles'
        // worth, rounded up to 16 bytes: still inside the block's field, whose
        // stride is a multiple of 64
        const long long cnt = tile_count(N, nreg);
        const long long pl = tile_point(N, nreg, (long long)nt.y + 127 < cnt ? (long long)nt.y + 127 : cnt - 1);
        const long long q0 = tile_point(N, nreg, nt.y);
        const long long nel = pl - q0 + 1 < 2 * 128 ? pl - q0 + 1 : 2 * 128;
        for (int r = threadIdx.x; r < D_SLOTS + 72; r += 32) {
          const char* a;
          int es;
          if (r < D_SLOTS) { a = (const char*)(D + N.doff + r * dfs + q0); es = sizeof(T); }
          else if (r < D_SLOTS + 24) { a = (const char*)(nin + (r - D_SLOTS) * fs + q0); es = sizeof(SI); }
          else if (r < D_SLOTS + 48) { a = (const char*)(N.tl[cur] + (r - D_SLOTS - 24) * fs + q0); es = 8; }
          else { a = (const char*)(N.K + (r - D_SLOTS - 48) * fs + q0); es = 8; }
          // the bulk prefetch wants a 16-byte aligned start and a multiple of 16
          // bytes: the row widened to 16-byte boundaries stays inside the field
          // row (its base is 256-byte aligned, its stride a multiple of 64)
          const size_t s0 = (size_t)a & ~(size_t)15;
          const size_t e0 = ((size_t)a + (size_t)nel * es + 15) & ~(size_t)15;
          asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(s0), "r"((unsigned)(e0 - s0)) : "memory");
        }
      }
     }
    }
#endif
    const long long p = tile_point(B, region, (long long)tile.y + threadIdx.x);
    if (p < 0) continue;
    const int cur = B.lvl[0];
    double* u0 = B.tl[cur];
    const SI* in = sub == 0 ? (const SI*)u0 : (const SI*)B.stage[sub == 2 ? 1 : 0];
    SO* out = sub == 3 ? (SO*)B.tl[(cur + 1) % 3] : (SO*)B.stage[sub == 1 ? 1 : 0];
    const double* in_side = sub == 0 ? nullptr : B.side[sub == 2 ? 1 : 0];
    auto q = make_pt<SI, SYMM>(in, B.b, p, in_side);
    EpiRK<T, SO> epi;
    epi.out_side = sub == 3 ? nullptr : B.side[sub == 1 ? 1 : 0];
    epi.u0 = u0;
    epi.K = B.K;
    epi.out = out;
    epi.fs = B.b.fs;
    epi.p = p;
    epi.sub = sub;
    epi.enforce = enforce != 0;
    epi.c = rk;
    epi.freeze = false;
    const int fm = B.b.face_mask;
    const bool on_face = ((fm & 1) && q.i == q.ex0 - 1) || ((fm & 2) && q.j == q.ex1 - 1) ||
                         ((fm & 4) && q.k == q.ex2 - 1) || ((fm & 8) && q.i == 0) || ((fm & 16) && q.j == 0) ||
                         ((fm & 32) && q.k == 0);
    // outer-face points are updated by k_face (a separate list), so no warp
    // here carries the Sommerfeld path for a few of its lanes
    if (on_face) continue;
    unsigned st;
    const PointGates G = point_gates(B.b, q.i, q.j, q.k);
    RhsAux aux{};
    if constexpr (SPLIT) {
      DPt<SI, SYMM, T> qd;
      static_cast<Pt<SI, SYMM>&>(qd) = q;
      qd.d = D + B.doff;
      qd.dfs = dfs;
      st = bssn_rhs_point<T, SI, SYMM, false, Z4C>(qd, B.C, G, aux, epi);
    } else {
      st = bssn_rhs_point<T, SI, SYMM, false, Z4C>(q, B.C, G, aux, epi);
    }
    if (st) atomicOr(status, st);
  }
}

// Outer-face points of a level (Sommerfeld on level 0, frozen on refined patch
// faces), one thread each, from the list faces[] = (block, point).
template <typename T, typename SI, typename SO, bool SYMM>
__global__ void __launch_bounds__(128) k_face(const StepBlock<T>* __restrict__ blocks, const int2* __restrict__ faces,
                                              int nfaces, int sub, RKConst rk, int enforce, unsigned* status) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nfaces; t += gridDim.x * blockDim.x) {
    const int2 fc = faces[t];
    const StepBlock<T>& B = blocks[fc.x];
    const long long p = fc.y;
    const int cur = B.lvl[0];
    double* u0 = B.tl[cur];
    const SI* in = sub == 0 ? (const SI*)u0 : (const SI*)B.stage[sub == 2 ? 1 : 0];
    auto q = make_pt<SI, SYMM>(in, B.b, p, sub == 0 ? nullptr : B.side[sub == 2 ? 1 : 0]);
    EpiRK<T, SO> epi;
    epi.out_side = sub == 3 ? nullptr : B.side[sub == 1 ? 1 : 0];
    epi.u0 = u0;
    epi.K = B.K;
    epi.out = sub == 3 ? (SO*)B.tl[(cur + 1) % 3] : (SO*)B.stage[sub == 1 ? 1 : 0];
    epi.fs = B.b.fs;
    epi.p = p;
    epi.sub = sub;
    epi.enforce = enforce != 0;
    epi.c = rk;
    epi.freeze = false;
    const unsigned st = face_point<T, SI, SO, SYMM>(B, q, epi);
    if (st) atomicOr(status, st);
  }
}

template <typename T, typename SS, bool SYMM>
cudaError_t launch_face(const void* blocks, const int2* faces, int nfaces, int sub, RKConst rk, int enforce,
                        unsigned* status, cudaStream_t s) {
  if (nfaces == 0) return cudaSuccess;
  const StepBlock<T>* bl = (const StepBlock<T>*)blocks;
  const int grid = (nfaces + 127) / 128 < 148 * 8 ? (nfaces + 127) / 128 : 148 * 8;
  if (sub == 0)
    k_face<T, double, SS, SYMM><<<grid, 128, 0, s>>>(bl, faces, nfaces, sub, rk, enforce, status);
  else if (sub == 3)
    k_face<T, SS, double, SYMM><<<grid, 128, 0, s>>>(bl, faces, nfaces, sub, rk, enforce, status);
  else
    k_face<T, SS, SS, SYMM><<<grid, 128, 0, s>>>(bl, faces, nfaces, sub, rk, enforce, status);
  return cudaGetLastError();
}

// SPLIT: the pointwise pass of the split form (per-thread loads over
// 128-point tiles); otherwise the fused kernel (128-point tiles).
template <typename T, typename SS, bool SYMM, bool SPLIT, bool Z4C>
cudaError_t launch_substep(const void* blocks, const int2* tiles, int ntiles, int sub, RKConst rk, int enforce,
                           unsigned* status, int grid, cudaStream_t s, const void* D, long long dfs) {
  const StepBlock<T>* bl = (const StepBlock<T>*)blocks;
  const T* d = (const T*)D;
  if (sub == 0)
    k_substep<T, double, SS, SYMM, SPLIT, Z4C><<<grid, 128, 0, s>>>(bl, tiles, ntiles, sub, rk, enforce, status, d, dfs);
  else if (sub == 3)
    k_substep<T, SS, double, SYMM, SPLIT, Z4C><<<grid, 128, 0, s>>>(bl, tiles, ntiles, sub, rk, enforce, status, d, dfs);
  else
    k_substep<T, SS, SS, SYMM, SPLIT, Z4C><<<grid, 128, 0, s>>>(bl, tiles, ntiles, sub, rk, enforce, status, d, dfs);
  return cudaGetLastError();
}

// Stencil pass launcher: substep 0 reads the FP64 state, 1-3 the stages;
// occ selects the compiled occupancy (0: two resident CTAs, 1: more).
template <typename T, typename SS>
cudaError_t launch_deriv(const void* blocks, const DerivItem* items, int nitems, int sub, void* D, long long dfs,
                         int grid, cudaStream_t s, int occ) {
  const StepBlock<T>* bl = (const StepBlock<T>*)blocks;
  // both < 48 KB: no opt-in attribute needed
  const size_t smem = occ ? kDerivSmem : kDerivSmemLow;
  constexpr int hi = sizeof(T) == 8 ? AMSS_DERIV_MINB_F64 : AMSS_DERIV_MINB_F32;
  if (sub == 0) {
    if (occ) k_deriv<T, double, hi><<<grid, DTHREADS, smem, s>>>(bl, items, nitems, sub, (T*)D, dfs);
    else k_deriv<T, double, kDerivMinbLow><<<grid, DTHREADS, smem, s>>>(bl, items, nitems, sub, (T*)D, dfs);
  } else {
    if (occ) k_deriv<T, SS, hi><<<grid, DTHREADS, smem, s>>>(bl, items, nitems, sub, (T*)D, dfs);
    else k_deriv<T, SS, kDerivMinbLow><<<grid, DTHREADS, smem, s>>>(bl, items, nitems, sub, (T*)D, dfs);
  }
  return cudaGetLastError();
}

// Drop-in RHS: all points of one block, RHS plus the diagnostic outputs.
template <bool SYMM>
__global__ void __launch_bounds__(128) k_rhs_dropin(BlockView b, Coefs<double> C, const double* __restrict__ u,
                                                    double* __restrict__ rhs, RhsAux aux, unsigned* status) {
  const long long n = (long long)b.ex[0] * b.ex[1] * b.ex[2];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    auto q = make_pt<double, SYMM>(u, b, p);
    const PointGates G = point_gates(b, q.i, q.j, q.k);
    EpiStore<double> epi{rhs, b.fs, p};
    const unsigned st = bssn_rhs_point<double, double, SYMM, true>(q, C, G, aux, epi);
    if (st) atomicOr(status, st);
  }
}

template <bool SYMM>
cudaError_t launch_rhs_dropin(int grid, cudaStream_t s, BlockView b, Coefs<double> C, const double* u, double* rhs,
                              RhsAux aux, unsigned* status) {
  k_rhs_dropin<SYMM><<<grid, 128, 0, s>>>(b, C, u, rhs, aux, status);
  return cudaGetLastError();
}

// Drop-in Z4c RHS: all points of one block, the 25 right-hand sides (the
// diagnostic outputs come from k_rhs_dropin, as ricci_gamma + constraint_bssn
// evaluate the BSSN formulas).
template <bool SYMM>
__global__ void __launch_bounds__(128) k_rhs_dropin_z4c(BlockView b, Coefs<double> C, const double* __restrict__ u,
                                                        double* __restrict__ rhs, const double* matter,
                                                        unsigned* status) {
  const long long n = (long long)b.ex[0] * b.ex[1] * b.ex[2];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    auto q = make_pt<double, SYMM>(u, b, p);
    const PointGates G = point_gates(b, q.i, q.j, q.k);
    EpiStore<double> epi{rhs, b.fs, p};
    RhsAux aux{};
    aux.matter = matter;
    aux.fs = b.fs;
    const unsigned st = bssn_rhs_point<double, double, SYMM, false, true>(q, C, G, aux, epi);
    if (st) atomicOr(status, st);
  }
}

template <bool SYMM>
cudaError_t launch_rhs_dropin_z4c(int grid, cudaStream_t s, BlockView b, Coefs<double> C, const double* u,
                                  double* rhs, const double* matter, unsigned* status) {
  k_rhs_dropin_z4c<SYMM><<<grid, 128, 0, s>>>(b, C, u, rhs, matter, status);
  return cudaGetLastError();
}

}  // namespace amss
