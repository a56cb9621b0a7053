// amss_common.cuh -- shared definitions of the B200 BSSN/Z4c evolution kernels.
//
// Layout in HBM: every grid function of a block is a Fortran-order array
// (i fastest) of ex0*ex1*ex2 values; the fields of one block sit at a fixed
// element stride `fs` from each other, so field f of a block starts at
// base + f*fs.  State order is the reference's (bssn_rhs.f90:6-11):
//   chi trK gxx gxy gxz gyy gyz gzz Axx Axy Axz Ayy Ayz Azz
//   Gamx Gamy Gamz Lap betax betay betaz dtSfx dtSfy dtSfz [TZ for Z4c]
// chi, Lap and the diagonal metric are stored as offsets (chi-1, alpha-1,
// g~ii-1), as the reference stores them.
#pragma once
#include <cstdint>
#ifndef AMSS_HOST_TRACE
#include <cuda_runtime.h>
#else
// host compile of the point functions for the adjoint generator (gen/)
#define __device__
#define __host__
#define __forceinline__ inline
template <typename T>
inline T __ldg(const T* p) { return *p; }
inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dsub_rn(double a, double b) { return a - b; }
inline double __dmul_rn(double a, double b) { return a * b; }
#endif

namespace amss {

enum Field : int {
  F_CHI = 0, F_TRK, F_GXX, F_GXY, F_GXZ, F_GYY, F_GYZ, F_GZZ,
  F_AXX, F_AXY, F_AXZ, F_AYY, F_AYZ, F_AZZ,
  F_GAMX, F_GAMY, F_GAMZ, F_LAP, F_BETAX, F_BETAY, F_BETAZ,
  F_DTSFX, F_DTSFY, F_DTSFZ, F_TZ, NFIELDS_BSSN = 24, NFIELDS_Z4C = 25
};

// Error bits of the device status word (mirrors the reference's NaN check,
// bssn_rhs.f90:110-138, plus the engine's own guards).
enum StatusBits : unsigned {
  ST_NAN = 1u,        // NaN in a checked input field
  ST_PINF = 2u,       // +inf seen in a checked input field
  ST_NINF = 4u,       // -inf seen in a checked input field
  ST_BAD_ARG = 8u,    // a kernel was handed an inconsistent descriptor
  ST_TIMEOUT = 16u,   // a bounded wait on an asynchronous copy gave up
};

// Parity of each state field under reflection x, y, z (bssn_class.C:177-330).
__host__ __device__ constexpr int soa_sign(int field, int dir) {
  // bit set = antisymmetric in that direction
  constexpr unsigned char anti[25] = {
      0, 0, 0, 3, 5, 0, 6, 0,   // chi trK gxx gxy gxz gyy gyz gzz
      0, 3, 5, 0, 6, 0,         // Axx .. Azz
      1, 2, 4, 0, 1, 2, 4,      // Gamx Gamy Gamz Lap betax betay betaz
      1, 2, 4, 0};              // dtSfx dtSfy dtSfz TZ
  return (anti[field] >> dir) & 1 ? -1 : 1;
}

// One block as the kernels see it.
struct BlockView {
  int ex[3];          // points per direction
  long long fs;       // element stride between fields
  const double* X;    // cell-centre coordinates, ex[0] values (device)
  const double* Y;    // ex[1] values
  const double* Z;    // ex[2] values
  double dx[3];       // X(2)-X(1), Y(2)-Y(1), Z(2)-Z(1), as the reference takes them
  int face_mask;      // bit d: outer face d (0:+x 1:+y 2:+z 3:-x 4:-y 5:-z) lies on the patch boundary
  int symmetry;       // 0 none, 1 equatorial, 2 octant
  int lowsym_mask;    // bit d: low side of direction d is a symmetry plane (imin = -ord)
};

}  // namespace amss
