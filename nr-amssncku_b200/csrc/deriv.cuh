// deriv.cuh -- the stencil pass of the split RK4 substep.
//
// One CTA takes one field of one (x, y) tile of a block (TX x TY points) and
// marches through z.  A ring of 7 z-planes of the tile plus a 3-cell halo sits
// in shared memory, filled as the reference's padded copy fh of
// symmetry_bd (fmisc.f90:877-901): cells at negative indices hold the mirrored
// value times the field's parity, cells past the block end are never read by
// the gated stencils and hold 0.  Each thread evaluates, for its point, the
// same gated stencils the per-point RHS would (diff_new.f90:946-1528,
// lopsidediff.f90:321-481, kodiss.f90:190-207) and stores them in the D slots
// of that field (stencil.cuh: dslots/doff); the pointwise pass reads them.
//
// Global traffic per field and point: one plane load amortised over the z
// march (~2.1 values per point for a 32 x 8 tile) instead of ~70 stencil loads.
#pragma once
#include "bssn_step.cuh"

namespace amss {

constexpr int DTX = 32, DTY = 8;            // tile of points per CTA
constexpr int DSX = DTX + 6, DSY = DTY + 6; // tile plus halo
constexpr int DPLANE = DSX * DSY;

struct DerivItem {
  int block;   // index into the level's StepBlock table
  int x0, y0;  // tile origin (array indices)
  int field;
};

// Shared-memory window with the interface of Pt (v / vpad).
template <typename A>
struct SmemPt {
  static constexpr bool kPre = false;
  using elem = A;
  const A* ring;
  int pl[7];       // plane offset of dk = -3 .. 3
  int li, lj;      // position in the tile
  int i, j, k;     // array indices
  long long p;
  template <typename T, int F>
  __device__ __forceinline__ T v(int di, int dj, int dk) const {
    return (T)ring[pl[dk + 3] + (lj + dj + 3) * DSX + (li + di + 3)];
  }
  template <typename T, int F>
  __device__ __forceinline__ T vpad(int di, int dj, int dk) const {
    return v<T, F>(di, dj, dk);
  }
};

// Load plane kk of field F of the stage input into ring slot `slot`.
template <int F, typename A, typename SI>
__device__ __forceinline__ void load_plane(A* ring, int slot, const SI* base, const double* side, long long fs,
                                           const int* ex, int x0, int y0, int kk) {
  A* dst = ring + slot * DPLANE;
  const long long sz = (long long)ex[0] * ex[1];
  bool negk = false;
  int k = kk;
  if (k < 0) { k = -k - 1; negk = soa_sign(F, 2) < 0; }
  const bool kin = k < ex[2];
  for (int t = threadIdx.x; t < DPLANE; t += blockDim.x) {
    const int a = t % DSX, b = t / DSX;
    int i = x0 - 3 + a, j = y0 - 3 + b;
    bool neg = negk;
    if (i < 0) { i = -i - 1; neg ^= (soa_sign(F, 0) < 0); }
    if (j < 0) { j = -j - 1; neg ^= (soa_sign(F, 1) < 0); }
    A v = A(0);
    if (kin && i < ex[0] && j < ex[1]) {
      const long long o = i + (long long)j * ex[0] + k * sz;
      if constexpr (sizeof(SI) == 4 && wide_field<F>()) v = (A)__ldg(side + side_slot(F) * fs + o);
      else v = (A)__ldg(base + F * fs + o);
      if (neg) v = -v;
    }
    dst[t] = v;
  }
}

template <typename T, int F, typename SI>
__device__ __forceinline__ void deriv_field(const StepBlock<T>& B, const SI* in, const double* in_side, int x0, int y0,
                                            T* D, long long dfs, unsigned char* smem) {
  using A = std::conditional_t<wide_field<F>(), double, T>;   // shared-memory and stencil type
  A* ring = reinterpret_cast<A*>(smem);
  const Coef<A>& C = pick<A>(B.C);
  const int* ex = B.b.ex;
  const int li = threadIdx.x % DTX, lj = threadIdx.x / DTX;
  const int i = x0 + li, j = y0 + lj;
  const bool mine = i < ex[0] && j < ex[1];
  const int fm = B.b.face_mask;
  T* d = D + B.doff;
  for (int m = 0; m < 6; ++m) load_plane<F, A>(ring, m, in, in_side, B.b.fs, ex, x0, y0, m - 3);
  for (int k = 0; k < ex[2]; ++k) {
    load_plane<F, A>(ring, (k + 6) % 7, in, in_side, B.b.fs, ex, x0, y0, k + 3);
    __syncthreads();
    const bool on_face = ((fm & 1) && i == ex[0] - 1) || ((fm & 2) && j == ex[1] - 1) ||
                         ((fm & 4) && k == ex[2] - 1) || ((fm & 8) && i == 0) || ((fm & 16) && j == 0) ||
                         ((fm & 32) && k == 0);
    if (mine && !on_face) {
      SmemPt<A> q;
      q.ring = ring;
      for (int m = 0; m < 7; ++m) q.pl[m] = ((k + m) % 7) * DPLANE;
      q.li = li;
      q.lj = lj;
      q.i = i;
      q.j = j;
      q.k = k;
      q.p = i + (long long)j * ex[0] + (long long)k * ex[0] * ex[1];
      const PointGates G = point_gates(B.b, i, j, k);
      constexpr int ns = dslots(F);
      constexpr int o = doff(F);
      const long long pp = q.p;
      if constexpr (ns == 11) {
        A fx, fy, fz, fxx, fxy, fxz, fyy, fyz, fzz;
        grad_a<A, F>(q, C, G.ord, fx, fy, fz);
        hess_a<A, F>(q, C, G.ord, fxx, fxy, fxz, fyy, fyz, fzz);
        d[(o + 0) * dfs + pp] = (T)fx; d[(o + 1) * dfs + pp] = (T)fy; d[(o + 2) * dfs + pp] = (T)fz;
        d[(o + 3) * dfs + pp] = (T)fxx; d[(o + 4) * dfs + pp] = (T)fxy; d[(o + 5) * dfs + pp] = (T)fxz;
        d[(o + 6) * dfs + pp] = (T)fyy; d[(o + 7) * dfs + pp] = (T)fyz; d[(o + 8) * dfs + pp] = (T)fzz;
      } else if constexpr (ns == 5) {
        A fx, fy, fz;
        grad_a<A, F>(q, C, G.ord, fx, fy, fz);
        d[(o + 0) * dfs + pp] = (T)fx; d[(o + 1) * dfs + pp] = (T)fy; d[(o + 2) * dfs + pp] = (T)fz;
      }
      // advection: beta at the point from the input (the shift is never a wide field)
      const long long cp = q.p;
      const T bx = (T)__ldg(in + F_BETAX * B.b.fs + cp);
      const T by = (T)__ldg(in + F_BETAY * B.b.fs + cp);
      const T bz = (T)__ldg(in + F_BETAZ * B.b.fs + cp);
      const A add1 = (F == F_GXX || F == F_GYY || F == F_GZZ) ? A(1) : A(0);
      A lop = A(0);
      if (G.lop) {
        Coefs<A> CC;
        CC.t = C;
        CC.d = pick<double>(B.C);
        lop = lop_dir<A, F, 0>(q, CC, lop, (A)bx, i, G.lo3[0], G.hi[0], add1);
        lop = lop_dir<A, F, 1>(q, CC, lop, (A)by, j, G.lo3[1], G.hi[1], add1);
        lop = lop_dir<A, F, 2>(q, CC, lop, (A)bz, k, G.lo3[2], G.hi[2], add1);
      }
      A ko = A(0);
      if (G.ko)
        ko = divh(ko_line<A, F, 0>(q), C.h[0]) + divh(ko_line<A, F, 1>(q), C.h[1]) + divh(ko_line<A, F, 2>(q), C.h[2]);
      d[(o + ns - 2) * dfs + pp] = (T)lop;
      d[(o + ns - 1) * dfs + pp] = (T)ko;
    }
    __syncthreads();
  }
}

// Stencil pass over a work list of (block, tile, field) items.
template <typename T, typename SI>
__global__ void __launch_bounds__(DTX * DTY) k_deriv(const StepBlock<T>* __restrict__ blocks,
                                                     const DerivItem* __restrict__ items, int nitems, int sub,
                                                     T* __restrict__ D, long long dfs) {
  extern __shared__ __align__(16) unsigned char smem[];
  for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
    const DerivItem it = items[w];
    const StepBlock<T>& B = blocks[it.block];
    const int cur = B.lvl[0];
    const SI* in = sub == 0 ? (const SI*)B.tl[cur] : (const SI*)B.stage[sub == 2 ? 1 : 0];
    const double* in_side = sub == 0 ? nullptr : B.side[sub == 2 ? 1 : 0];
    switch (it.field) {
#define AMSS_DF(F) case F: deriv_field<T, F, SI>(B, in, in_side, it.x0, it.y0, D, dfs, smem); break;
      AMSS_DF(F_CHI) AMSS_DF(F_TRK) AMSS_DF(F_GXX) AMSS_DF(F_GXY) AMSS_DF(F_GXZ) AMSS_DF(F_GYY)
      AMSS_DF(F_GYZ) AMSS_DF(F_GZZ) AMSS_DF(F_AXX) AMSS_DF(F_AXY) AMSS_DF(F_AXZ) AMSS_DF(F_AYY)
      AMSS_DF(F_AYZ) AMSS_DF(F_AZZ) AMSS_DF(F_GAMX) AMSS_DF(F_GAMY) AMSS_DF(F_GAMZ) AMSS_DF(F_LAP)
      AMSS_DF(F_BETAX) AMSS_DF(F_BETAY) AMSS_DF(F_BETAZ) AMSS_DF(F_DTSFX) AMSS_DF(F_DTSFY) AMSS_DF(F_DTSFZ)
#undef AMSS_DF
      default: break;
    }
    __syncthreads();
  }
}

}  // namespace amss
