// substep_common.cuh -- point indexing, the global-memory point accessor and
// the outer-face point update shared by the RK4 substep kernels.
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

// Outer-face point of a block: the NaN check of the input, then the
// Sommerfeld RHS (level 0, sommerfeld_rout.f90:223-449) or the frozen value
// (refined patch faces, sommerfeld_rout.f90:122-139); epilogue included.
template <typename T, typename SI, typename SO, bool SYMM>
__device__ __forceinline__ unsigned face_point(const StepBlock<T>& B, const Pt<SI, SYMM>& q, EpiRK<T, SO>& epi) {
  unsigned st;
  // NaN check of the input, as the full RHS would do it
  T chk[25];
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
  if (B.nf == NFIELDS_Z4C) {  // Z4c_rhs.f90:230-262 also checks B^i and Theta
    chk[21] = q.template v<T, F_DTSFX>(0, 0, 0); chk[22] = q.template v<T, F_DTSFY>(0, 0, 0);
    chk[23] = q.template v<T, F_DTSFZ>(0, 0, 0); chk[24] = q.template v<T, F_TZ>(0, 0, 0);
    st = nan_bits(chk, 25);
  } else {
    st = nan_bits(chk, 21);
  }
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
    if (B.nf == NFIELDS_Z4C) AMSS_SOMM(F_TZ, v1)   // Theta: propspeed 1, parity (+,+,+)
#undef AMSS_SOMM
  } else {
    epi.freeze = true;
#define AMSS_FRZ(F) epi.template put<F>(T(0));
    AMSS_FRZ(F_CHI) AMSS_FRZ(F_TRK) AMSS_FRZ(F_GXX) AMSS_FRZ(F_GXY) AMSS_FRZ(F_GXZ) AMSS_FRZ(F_GYY)
    AMSS_FRZ(F_GYZ) AMSS_FRZ(F_GZZ) AMSS_FRZ(F_AXX) AMSS_FRZ(F_AXY) AMSS_FRZ(F_AXZ) AMSS_FRZ(F_AYY)
    AMSS_FRZ(F_AYZ) AMSS_FRZ(F_AZZ) AMSS_FRZ(F_GAMX) AMSS_FRZ(F_GAMY) AMSS_FRZ(F_GAMZ) AMSS_FRZ(F_LAP)
    AMSS_FRZ(F_BETAX) AMSS_FRZ(F_BETAY) AMSS_FRZ(F_BETAZ) AMSS_FRZ(F_DTSFX) AMSS_FRZ(F_DTSFY)
    AMSS_FRZ(F_DTSFZ)
    if (B.nf == NFIELDS_Z4C) AMSS_FRZ(F_TZ)
#undef AMSS_FRZ
  }
  epi.finish();
  return st;
}

}  // namespace amss
