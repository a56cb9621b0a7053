// substep_impl.cuh -- the fused RK4 substep kernel template and its launcher.
// Instantiated in one translation unit per (precision, symmetry) pair so the
// large kernels compile in parallel.
#pragma once
#include "deriv.cuh"

namespace amss {

__device__ __forceinline__ void point_ijk(long long p, const int* ex, int& i, int& j, int& k) {
  const long long s1 = (long long)ex[0] * ex[1];
  k = (int)(p / s1);
  const long long r = p - (long long)k * s1;
  j = (int)(r / ex[0]);
  i = (int)(r - (long long)j * ex[0]);
}

template <typename SI, bool SYMM>
__device__ __forceinline__ Pt<SI, SYMM> make_pt(const SI* base, const BlockView& b, long long p,
                                               const double* side = nullptr) {
  Pt<SI, SYMM> q;
  q.base = base;
  q.side = side;
  q.fs = b.fs;
  q.p = p;
  q.sy = b.ex[0];
  q.sz = (long long)b.ex[0] * b.ex[1];
  point_ijk(p, b.ex, q.i, q.j, q.k);
  q.ex0 = b.ex[0];
  q.ex1 = b.ex[1];
  q.ex2 = b.ex[2];
  return q;
}

// Fused RK4 substep over a tile list of one level.  Substep `sub` reads
// (sub0: u0, sub1: A, sub2: B, sub3: A) and writes (A, B, A, unew).
// SPLIT: the stencil terms come from the D array the stencil pass (k_deriv)
// wrote for this substep; otherwise every stencil is evaluated here.
template <typename T, typename SI, typename SO, bool SYMM, bool SPLIT>
__global__ void __launch_bounds__(128) k_substep(const StepBlock<T>* __restrict__ blocks, const int2* __restrict__ tiles,
                                                 int ntiles, int sub, RKConst rk, int enforce, unsigned* status,
                                                 const T* __restrict__ D, long long dfs) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 tile = tiles[t];
    const StepBlock<T>& B = blocks[tile.x];
    const long long p = (long long)tile.y + threadIdx.x;
    if (p >= B.npts) continue;
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
    unsigned st = 0;
    if (!on_face) {
      const PointGates G = point_gates(B.b, q.i, q.j, q.k);
      RhsAux aux{};
      if constexpr (SPLIT) {
        DPt<SI, SYMM, T> qd;
        static_cast<Pt<SI, SYMM>&>(qd) = q;
        qd.d = D + B.doff;
        qd.dfs = dfs;
        st = bssn_rhs_point<T, SI, SYMM, false>(qd, B.C, G, aux, epi);
      } else {
        st = bssn_rhs_point<T, SI, SYMM, false>(q, B.C, G, aux, epi);
      }
    } else {
      // NaN check of the input, as the full RHS would do it
      T chk[21];
      chk[0] = q.template v<T, F_CHI>(0, 0, 0); chk[1] = q.template v<T, F_TRK>(0, 0, 0);
      chk[2] = q.template v<T, F_GXX>(0, 0, 0); chk[3] = q.template v<T, F_GXY>(0, 0, 0);
      chk[4] = q.template v<T, F_GXZ>(0, 0, 0); chk[5] = q.template v<T, F_GYY>(0, 0, 0);
      chk[6] = q.template v<T, F_GYZ>(0, 0, 0); chk[7] = q.template v<T, F_GZZ>(0, 0, 0);
      chk[8] = q.template v<T, F_AXX>(0, 0, 0); chk[9] = q.template v<T, F_AXY>(0, 0, 0);
      chk[10] = q.template v<T, F_AXZ>(0, 0, 0); chk[11] = q.template v<T, F_AYY>(0, 0, 0);
      chk[12] = q.template v<T, F_AYZ>(0, 0, 0); chk[13] = q.template v<T, F_AZZ>(0, 0, 0);
      chk[14] = q.template v<T, F_GAMX>(0, 0, 0); chk[15] = q.template v<T, F_GAMY>(0, 0, 0);
      chk[16] = q.template v<T, F_GAMZ>(0, 0, 0); chk[17] = q.template v<T, F_LAP>(0, 0, 0);
      chk[18] = q.template v<T, F_BETAX>(0, 0, 0); chk[19] = q.template v<T, F_BETAY>(0, 0, 0);
      chk[20] = q.template v<T, F_BETAZ>(0, 0, 0);
      st = nan_bits(chk, 21);
      if (B.lev0) {
        const T x = (T)B.b.X[q.i], y = (T)B.b.Y[q.j], z = (T)B.b.Z[q.k];
        int lo[3], hi[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          lo[d] = ((B.b.lowsym_mask >> d) & 1) ? -1 : 0;
          hi[d] = B.b.ex[d] - 1;
        }
        const T v2 = T(1.4142135623730951), v1 = T(1);
#define AMSS_SOMM(F, V) epi.template put<F>(sommerfeld_point<T, F>(q, B.d2s, lo, hi, x, y, z, V));
        AMSS_SOMM(F_CHI, v2) AMSS_SOMM(F_TRK, v2) AMSS_SOMM(F_GXX, v1) AMSS_SOMM(F_GXY, v1)
        AMSS_SOMM(F_GXZ, v1) AMSS_SOMM(F_GYY, v1) AMSS_SOMM(F_GYZ, v1) AMSS_SOMM(F_GZZ, v1)
        AMSS_SOMM(F_AXX, v1) AMSS_SOMM(F_AXY, v1) AMSS_SOMM(F_AXZ, v1) AMSS_SOMM(F_AYY, v1)
        AMSS_SOMM(F_AYZ, v1) AMSS_SOMM(F_AZZ, v1) AMSS_SOMM(F_GAMX, v1) AMSS_SOMM(F_GAMY, v1)
        AMSS_SOMM(F_GAMZ, v1) AMSS_SOMM(F_LAP, v2) AMSS_SOMM(F_BETAX, v1) AMSS_SOMM(F_BETAY, v1)
        AMSS_SOMM(F_BETAZ, v1) AMSS_SOMM(F_DTSFX, v1) AMSS_SOMM(F_DTSFY, v1) AMSS_SOMM(F_DTSFZ, v1)
#undef AMSS_SOMM
      } else {
        epi.freeze = true;
#define AMSS_FRZ(F) epi.template put<F>(T(0));
        AMSS_FRZ(F_CHI) AMSS_FRZ(F_TRK) AMSS_FRZ(F_GXX) AMSS_FRZ(F_GXY) AMSS_FRZ(F_GXZ) AMSS_FRZ(F_GYY)
        AMSS_FRZ(F_GYZ) AMSS_FRZ(F_GZZ) AMSS_FRZ(F_AXX) AMSS_FRZ(F_AXY) AMSS_FRZ(F_AXZ) AMSS_FRZ(F_AYY)
        AMSS_FRZ(F_AYZ) AMSS_FRZ(F_AZZ) AMSS_FRZ(F_GAMX) AMSS_FRZ(F_GAMY) AMSS_FRZ(F_GAMZ) AMSS_FRZ(F_LAP)
        AMSS_FRZ(F_BETAX) AMSS_FRZ(F_BETAY) AMSS_FRZ(F_BETAZ) AMSS_FRZ(F_DTSFX) AMSS_FRZ(F_DTSFY)
        AMSS_FRZ(F_DTSFZ)
#undef AMSS_FRZ
      }
      epi.finish();
    }
    if (st) atomicOr(status, st);
  }
}

template <typename T, typename SS, bool SYMM, bool SPLIT>
cudaError_t launch_substep(const void* blocks, const int2* tiles, int ntiles, int sub, RKConst rk, int enforce,
                           unsigned* status, int grid, cudaStream_t s, const void* D, long long dfs) {
  const StepBlock<T>* bl = (const StepBlock<T>*)blocks;
  const T* d = (const T*)D;
  if (sub == 0)
    k_substep<T, double, SS, SYMM, SPLIT><<<grid, 128, 0, s>>>(bl, tiles, ntiles, sub, rk, enforce, status, d, dfs);
  else if (sub == 3)
    k_substep<T, SS, double, SYMM, SPLIT><<<grid, 128, 0, s>>>(bl, tiles, ntiles, sub, rk, enforce, status, d, dfs);
  else
    k_substep<T, SS, SS, SYMM, SPLIT><<<grid, 128, 0, s>>>(bl, tiles, ntiles, sub, rk, enforce, status, d, dfs);
  return cudaGetLastError();
}

// Stencil pass launcher: substep 0 reads the FP64 state, 1-3 the stages.
template <typename T, typename SS>
cudaError_t launch_deriv(const void* blocks, const DerivItem* items, int nitems, int sub, void* D, long long dfs,
                         int grid, cudaStream_t s) {
  const StepBlock<T>* bl = (const StepBlock<T>*)blocks;
  const size_t smem = 7 * DPLANE * sizeof(double);
  if (sub == 0) {
    cudaFuncSetAttribute(k_deriv<T, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_deriv<T, double><<<grid, DTX * DTY, smem, s>>>(bl, items, nitems, sub, (T*)D, dfs);
  } else {
    cudaFuncSetAttribute(k_deriv<T, SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_deriv<T, SS><<<grid, DTX * DTY, smem, s>>>(bl, items, nitems, sub, (T*)D, dfs);
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

}  // namespace amss
