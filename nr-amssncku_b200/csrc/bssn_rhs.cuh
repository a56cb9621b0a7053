// bssn_rhs.cuh -- the BSSN right-hand side at one grid point.
//
// Restates compute_rhs_bssn (bssn_rhs.f90:5-1184, GAUGE 0, Cell,
// ghost_width 3) for a single point: every derivative the Fortran takes as a
// whole-array stencil pass is taken here at the point itself, and every
// pointwise statement keeps the Fortran's association order.  Each evolved
// field is finished -- pointwise value, + lopsided advection x, y, z, + KO
// dissipation, in that order as bssn_rhs.f90:948-1042 adds them -- as soon as
// its pointwise value is known and handed to the epilogue `E`, which either
// stores it (the per-block RHS entry point) or applies the RK4 substep update
// in place of the store (the fused evolution step).  That keeps the number of
// live values per thread, and so register spills, down.
//
// T  : arithmetic type (double for the FP64 form, float for the mixed form)
// SI : storage type of the stencil input (double or float)
#pragma once
#include "stencil.cuh"

namespace amss {

struct RhsAux {                     // optional diagnostic outputs (drop-in entry)
  double* gamma;                    // 18 fields: physical Christoffel symbols
  double* ricci;                    // 6 fields: physical Ricci tensor
  double* cons;                     // 7 fields: ham, movx..z, Gmx..z (co == 0)
  const double* matter;             // 10 fields: rho Sx Sy Sz Sxx Sxy Sxz Syy Syz Szz
  long long fs;                     // field stride of these arrays
  int co;                           // 0: compute constraints
};

struct PointGates {
  int ord;          // derivative order gate: 2 (4th order), 1 (2nd order), 0 (zero)
  bool ko;          // KO applies (all +-3 fit)
  bool lop;         // point is inside the lopsided loop (all indices <= ex-2)
  int lo3[3];       // lopsided imin, 0-based
  int hi[3];        // imax, 0-based
};

__device__ __forceinline__ PointGates point_gates(const BlockView& b, int i, int j, int k) {
  PointGates g;
  const int id[3] = {i, j, k};
  bool o4 = true, o2 = true, ko = true, lp = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const bool ls = (b.lowsym_mask >> d) & 1;
    const int lo2 = ls ? -2 : 0, lo3 = ls ? -3 : 0, hi = b.ex[d] - 1;
    o4 = o4 && (id[d] - 2 >= lo2) && (id[d] + 2 <= hi);
    o2 = o2 && (id[d] - 1 >= lo2) && (id[d] + 1 <= hi);
    ko = ko && (id[d] - 3 >= lo3) && (id[d] + 3 <= hi);
    lp = lp && (id[d] <= hi - 1);
    g.lo3[d] = lo3;
    g.hi[d] = hi;
  }
  g.ord = o4 ? 2 : (o2 ? 1 : 0);
  g.ko = ko;
  g.lop = lp;
  return g;
}

// Finish one field: + lopsided (x, y, z) + KO, then hand it to the epilogue.
// `add1` = 1 for the diagonal metric (advected as g = d + 1, bssn_rhs.f90:948-953).
// KO1: dissipate f + add1 rather than f (the Z4c diagonal metric).
template <typename T, int F, bool KO1 = false, typename P, typename E>
__device__ __forceinline__ void finish_field(const P& q, const Coefs<T>& C, const PointGates& g, T r, T bx, T by,
                                             T bz, T add1, E& epi) {
  if constexpr (P::kPre) {
    // split form: the stencil pass stored advection + KO (0 where neither applies)
    r = r + q.template dv<T>(doff(F) + dslots(F) - 1);
    epi.template put<F>(r);
  } else {
    if (g.lop) {
      r = lop_dir<T, F, 0>(q, C, r, bx, q.i, g.lo3[0], g.hi[0], add1);
      r = lop_dir<T, F, 1>(q, C, r, by, q.j, g.lo3[1], g.hi[1], add1);
      r = lop_dir<T, F, 2>(q, C, r, bz, q.k, g.lo3[2], g.hi[2], add1);
    }
    if (g.ko) {
      using A = std::conditional_t<wide_field<F>(), double, T>;
      const Coef<A>& c = pick<A>(C);
      auto kx = [&](int o) { return q.template v<A, F>(o, 0, 0); };
      auto ky = [&](int o) { return q.template v<A, F>(0, o, 0); };
      auto kz = [&](int o) { return q.template v<A, F>(0, 0, o); };
      const A ks = kodiv(ko_sum_rn<A, KO1>(kx), c, 0) + kodiv(ko_sum_rn<A, KO1>(ky), c, 1) +
                   kodiv(ko_sum_rn<A, KO1>(kz), c, 2);
      r = r + (T)(c.ko * ks);
    }
    epi.template put<F>(r);
  }
}

// NaN check of bssn_rhs.f90:110-138 on the point's own 21 checked values.
template <typename T>
__device__ __forceinline__ unsigned nan_bits(const T* v, int n) {
  unsigned s = 0;
  for (int m = 0; m < n; ++m) {
    const T x = v[m];
    if (x != x) s |= ST_NAN;
    else if (isinf(x)) s |= (x > T(0)) ? ST_PINF : ST_NINF;
  }
  return s;
}

// Z4C: the Z4c right-hand side of Z4c_rhs.f90:126-1295 (25 fields, Theta
// last; kappa1 = 0.02, kappa2 = 0 from cpbc.f90:5-20) instead of BSSN.
// Epilogues with a member ham(T) receive the Hamiltonian constraint.
template <typename E, typename = void>
struct epi_wants_ham : std::false_type {};
template <typename E>
struct epi_wants_ham<E, std::void_t<decltype(&E::ham)>> : std::true_type {};

// Type of the FP64 centre values of chi and alpha: double for the FP32 and
// FP64 forms; a recording scalar type (the adjoint generator) maps to itself.
template <typename T>
struct wide {
  using type = double;
};
template <typename T>
using wide_t = typename wide<T>::type;

template <typename T, typename SI, bool SYMM, bool AUX, bool Z4C = false, typename E, typename P>
__device__ __forceinline__ unsigned bssn_rhs_point(const P& q, const Coefs<T>& C, const PointGates& G,
                                                   const RhsAux& aux, E& epi) {
  static_assert(!(AUX && P::kPre), "the diagnostic outputs need the stencil accessor");
  static_assert(!(AUX && Z4C), "Z4c diagnostics come from the BSSN diagnostic pass");
  const T kappa1 = T(0.02), kappa2 = T(0);
  const T ZEO = T(0), ONE = T(1), TWO = T(2), FOUR = T(4), EIGHT = T(8), HALF = T(0.5);
  const T FF = T(0.75), eta = T(2);
  const T F1o3 = T(1.0 / 3.0), F2o3 = T(2.0 / 3.0), F3o2 = T(1.5);
  const T PI = T(3.141592653589793238462643383279502884);
  const int ord = G.ord;

  // centre values; chi and alpha are read and shifted in FP64 (chi -> 0 near a
  // puncture, so chi+1 must be formed before rounding to T)
  using W = wide_t<T>;
  const W chi64 = q.template v<W, F_CHI>(0, 0, 0), Lap64 = q.template v<W, F_LAP>(0, 0, 0);
  const T chi = (T)chi64, trK = q.template v<T, F_TRK>(0, 0, 0);
  const T dxx = q.template v<T, F_GXX>(0, 0, 0), gxy = q.template v<T, F_GXY>(0, 0, 0);
  const T gxz = q.template v<T, F_GXZ>(0, 0, 0), dyy = q.template v<T, F_GYY>(0, 0, 0);
  const T gyz = q.template v<T, F_GYZ>(0, 0, 0), dzz = q.template v<T, F_GZZ>(0, 0, 0);
  const T Axx = q.template v<T, F_AXX>(0, 0, 0), Axy = q.template v<T, F_AXY>(0, 0, 0);
  const T Axz = q.template v<T, F_AXZ>(0, 0, 0), Ayy = q.template v<T, F_AYY>(0, 0, 0);
  const T Ayz = q.template v<T, F_AYZ>(0, 0, 0), Azz = q.template v<T, F_AZZ>(0, 0, 0);
  const T Gamx = q.template v<T, F_GAMX>(0, 0, 0), Gamy = q.template v<T, F_GAMY>(0, 0, 0);
  const T Gamz = q.template v<T, F_GAMZ>(0, 0, 0), Lap = (T)Lap64;
  const T betax = q.template v<T, F_BETAX>(0, 0, 0), betay = q.template v<T, F_BETAY>(0, 0, 0);
  const T betaz = q.template v<T, F_BETAZ>(0, 0, 0);
  const T dtSfx = q.template v<T, F_DTSFX>(0, 0, 0), dtSfy = q.template v<T, F_DTSFY>(0, 0, 0);
  const T dtSfz = q.template v<T, F_DTSFZ>(0, 0, 0);
  T TZ = ZEO;
  if constexpr (Z4C) TZ = q.template v<T, F_TZ>(0, 0, 0);
  unsigned status;
  if constexpr (Z4C) {  // Z4c_rhs.f90:230-262 checks 25 fields
    const T chk[25] = {chi, trK, dxx, gxy, gxz, dyy, gyz, dzz, Axx, Axy, Axz, Ayy, Ayz, Azz,
                       Gamx, Gamy, Gamz, Lap, betax, betay, betaz, dtSfx, dtSfy, dtSfz, TZ};
    status = nan_bits(chk, 25);
  } else {
    const T chk[21] = {chi, trK, dxx, gxy, gxz, dyy, gyz, dzz, Axx, Axy, Axz, Ayy, Ayz, Azz,
                       Gamx, Gamy, Gamz, Lap, betax, betay, betaz};
    status = nan_bits(chk, 21);
  }
  // Z4c: K + 2 Theta wherever the evolution uses the trace (Z4c_rhs.f90:277)
  const T trKd = Z4C ? trK + TWO * TZ : trK;

  // matter (zero in vacuum: the engine passes no matter fields)
  T rho = ZEO, Sx = ZEO, Sy = ZEO, Sz = ZEO, Sxx = ZEO, Sxy = ZEO, Sxz = ZEO, Syy = ZEO, Syz = ZEO, Szz = ZEO;
  {
    if (aux.matter) {
      const double* m = aux.matter + q.p;
      rho = (T)m[0]; Sx = (T)m[aux.fs]; Sy = (T)m[2 * aux.fs]; Sz = (T)m[3 * aux.fs];
      Sxx = (T)m[4 * aux.fs]; Sxy = (T)m[5 * aux.fs]; Sxz = (T)m[6 * aux.fs];
      Syy = (T)m[7 * aux.fs]; Syz = (T)m[8 * aux.fs]; Szz = (T)m[9 * aux.fs];
    }
  }

  const T alpn1 = (T)(Lap64 + W(1.0)), chin1 = (T)(chi64 + W(1.0));
  const T gxx = dxx + ONE, gyy = dyy + ONE, gzz = dzz + ONE;

  // :152-160
  T betaxx, betaxy, betaxz, betayx, betayy, betayz, betazx, betazy, betazz;
  grad<T, F_BETAX>(q, C, ord, betaxx, betaxy, betaxz);
  grad<T, F_BETAY>(q, C, ord, betayx, betayy, betayz);
  grad<T, F_BETAZ>(q, C, ord, betazx, betazy, betazz);
  const T div_beta = betaxx + betayy + betazz;
  T chix, chiy, chiz;
  grad<T, F_CHI>(q, C, ord, chix, chiy, chiz);
  finish_field<T, F_CHI>(q, C, G, F2o3 * chin1 * (alpn1 * trKd - div_beta), betax, betay, betaz, ZEO, epi);

  // :791-795 gauge pieces that need nothing else
  finish_field<T, F_LAP>(q, C, G, -TWO * alpn1 * trK, betax, betay, betaz, ZEO, epi);
  finish_field<T, F_BETAX>(q, C, G, FF * dtSfx, betax, betay, betaz, ZEO, epi);
  finish_field<T, F_BETAY>(q, C, G, FF * dtSfy, betax, betay, betaz, ZEO, epi);
  finish_field<T, F_BETAZ>(q, C, G, FF * dtSfz, betax, betay, betaz, ZEO, epi);

  // :162-191
  T gxxx, gxxy, gxxz, gxyx, gxyy, gxyz, gxzx, gxzy, gxzz, gyyx, gyyy, gyyz, gyzx, gyzy, gyzz, gzzx, gzzy, gzzz;
  grad<T, F_GXX>(q, C, ord, gxxx, gxxy, gxxz);
  grad<T, F_GXY>(q, C, ord, gxyx, gxyy, gxyz);
  grad<T, F_GXZ>(q, C, ord, gxzx, gxzy, gxzz);
  grad<T, F_GYY>(q, C, ord, gyyx, gyyy, gyyz);
  grad<T, F_GYZ>(q, C, ord, gyzx, gyzy, gyzz);
  grad<T, F_GZZ>(q, C, ord, gzzx, gzzy, gzzz);

  finish_field<T, F_GXX, Z4C>(q, C, G,
                         -TWO * alpn1 * Axx - F2o3 * gxx * div_beta +
                             TWO * (gxx * betaxx + gxy * betayx + gxz * betazx),
                         betax, betay, betaz, ONE, epi);
  finish_field<T, F_GYY, Z4C>(q, C, G,
                         -TWO * alpn1 * Ayy - F2o3 * gyy * div_beta +
                             TWO * (gxy * betaxy + gyy * betayy + gyz * betazy),
                         betax, betay, betaz, ONE, epi);
  finish_field<T, F_GZZ, Z4C>(q, C, G,
                         -TWO * alpn1 * Azz - F2o3 * gzz * div_beta +
                             TWO * (gxz * betaxz + gyz * betayz + gzz * betazz),
                         betax, betay, betaz, ONE, epi);
  finish_field<T, F_GXY>(q, C, G,
                         -TWO * alpn1 * Axy + F1o3 * gxy * div_beta + gxx * betaxy + gxz * betazy +
                             gyy * betayx + gyz * betazx - gxy * betazz,
                         betax, betay, betaz, ZEO, epi);
  finish_field<T, F_GYZ>(q, C, G,
                         -TWO * alpn1 * Ayz + F1o3 * gyz * div_beta + gxy * betaxz + gyy * betayz +
                             gxz * betaxy + gzz * betazy - gyz * betaxx,
                         betax, betay, betaz, ZEO, epi);
  finish_field<T, F_GXZ>(q, C, G,
                         -TWO * alpn1 * Axz + F1o3 * gxz * div_beta + gxx * betaxz + gxy * betayz +
                             gyz * betayx + gzz * betazx - gxz * betayy,
                         betax, betay, betaz, ZEO, epi);

  // :194-201 invert the conformal metric
  T gupzz = gxx * gyy * gzz + gxy * gyz * gxz + gxz * gxy * gyz - gxz * gyy * gxz - gxy * gxy * gzz -
            gxx * gyz * gyz;
  const T gupxx = (gyy * gzz - gyz * gyz) / gupzz;
  const T gupxy = -(gxy * gzz - gyz * gxz) / gupzz;
  const T gupxz = (gxy * gyz - gyy * gxz) / gupzz;
  const T gupyy = (gxx * gzz - gxz * gxz) / gupzz;
  const T gupyz = -(gxx * gyz - gxy * gxz) / gupzz;
  gupzz = (gxx * gyy - gxy * gxy) / gupzz;

  if constexpr (AUX) {
    if (aux.co == 0) {  // :203-232
      double* o = aux.cons + q.p;
      o[4 * aux.fs] = (double)(Gamx - (gupxx * (gupxx * gxxx + gupxy * gxyx + gupxz * gxzx) +
                                       gupxy * (gupxx * gxyx + gupxy * gyyx + gupxz * gyzx) +
                                       gupxz * (gupxx * gxzx + gupxy * gyzx + gupxz * gzzx) +
                                       gupxx * (gupxy * gxxy + gupyy * gxyy + gupyz * gxzy) +
                                       gupxy * (gupxy * gxyy + gupyy * gyyy + gupyz * gyzy) +
                                       gupxz * (gupxy * gxzy + gupyy * gyzy + gupyz * gzzy) +
                                       gupxx * (gupxz * gxxz + gupyz * gxyz + gupzz * gxzz) +
                                       gupxy * (gupxz * gxyz + gupyz * gyyz + gupzz * gyzz) +
                                       gupxz * (gupxz * gxzz + gupyz * gyzz + gupzz * gzzz)));
      o[5 * aux.fs] = (double)(Gamy - (gupxx * (gupxy * gxxx + gupyy * gxyx + gupyz * gxzx) +
                                       gupxy * (gupxy * gxyx + gupyy * gyyx + gupyz * gyzx) +
                                       gupxz * (gupxy * gxzx + gupyy * gyzx + gupyz * gzzx) +
                                       gupxy * (gupxy * gxxy + gupyy * gxyy + gupyz * gxzy) +
                                       gupyy * (gupxy * gxyy + gupyy * gyyy + gupyz * gyzy) +
                                       gupyz * (gupxy * gxzy + gupyy * gyzy + gupyz * gzzy) +
                                       gupxy * (gupxz * gxxz + gupyz * gxyz + gupzz * gxzz) +
                                       gupyy * (gupxz * gxyz + gupyz * gyyz + gupzz * gyzz) +
                                       gupyz * (gupxz * gxzz + gupyz * gyzz + gupzz * gzzz)));
      o[6 * aux.fs] = (double)(Gamz - (gupxx * (gupxz * gxxx + gupyz * gxyx + gupzz * gxzx) +
                                       gupxy * (gupxz * gxyx + gupyz * gyyx + gupzz * gyzx) +
                                       gupxz * (gupxz * gxzx + gupyz * gyzx + gupzz * gzzx) +
                                       gupxy * (gupxz * gxxy + gupyz * gxyy + gupzz * gxzy) +
                                       gupyy * (gupxz * gxyy + gupyz * gyyy + gupzz * gyzy) +
                                       gupyz * (gupxz * gxzy + gupyz * gyzy + gupzz * gzzy) +
                                       gupxz * (gupxz * gxxz + gupyz * gxyz + gupzz * gxzz) +
                                       gupyz * (gupxz * gxyz + gupyz * gyyz + gupzz * gyzz) +
                                       gupzz * (gupxz * gxzz + gupyz * gyzz + gupzz * gzzz)));
    }
  }

  // :235-257 conformal Christoffel symbols of the second kind
  T Gamxxx = HALF * (gupxx * gxxx + gupxy * (TWO * gxyx - gxxy) + gupxz * (TWO * gxzx - gxxz));
  T Gamyxx = HALF * (gupxy * gxxx + gupyy * (TWO * gxyx - gxxy) + gupyz * (TWO * gxzx - gxxz));
  T Gamzxx = HALF * (gupxz * gxxx + gupyz * (TWO * gxyx - gxxy) + gupzz * (TWO * gxzx - gxxz));
  T Gamxyy = HALF * (gupxx * (TWO * gxyy - gyyx) + gupxy * gyyy + gupxz * (TWO * gyzy - gyyz));
  T Gamyyy = HALF * (gupxy * (TWO * gxyy - gyyx) + gupyy * gyyy + gupyz * (TWO * gyzy - gyyz));
  T Gamzyy = HALF * (gupxz * (TWO * gxyy - gyyx) + gupyz * gyyy + gupzz * (TWO * gyzy - gyyz));
  T Gamxzz = HALF * (gupxx * (TWO * gxzz - gzzx) + gupxy * (TWO * gyzz - gzzy) + gupxz * gzzz);
  T Gamyzz = HALF * (gupxy * (TWO * gxzz - gzzx) + gupyy * (TWO * gyzz - gzzy) + gupyz * gzzz);
  T Gamzzz = HALF * (gupxz * (TWO * gxzz - gzzx) + gupyz * (TWO * gyzz - gzzy) + gupzz * gzzz);
  T Gamxxy = HALF * (gupxx * gxxy + gupxy * gyyx + gupxz * (gxzy + gyzx - gxyz));
  T Gamyxy = HALF * (gupxy * gxxy + gupyy * gyyx + gupyz * (gxzy + gyzx - gxyz));
  T Gamzxy = HALF * (gupxz * gxxy + gupyz * gyyx + gupzz * (gxzy + gyzx - gxyz));
  T Gamxxz = HALF * (gupxx * gxxz + gupxy * (gxyz + gyzx - gxzy) + gupxz * gzzx);
  T Gamyxz = HALF * (gupxy * gxxz + gupyy * (gxyz + gyzx - gxzy) + gupyz * gzzx);
  T Gamzxz = HALF * (gupxz * gxxz + gupyz * (gxyz + gyzx - gxzy) + gupzz * gzzx);
  T Gamxyz = HALF * (gupxx * (gxyz + gxzy - gyzx) + gupxy * gyyz + gupxz * gzzy);
  T Gamyyz = HALF * (gupxy * (gxyz + gxzy - gyzx) + gupyy * gyyz + gupyz * gzzy);
  T Gamzyz = HALF * (gupxz * (gxyz + gxzy - gyzx) + gupyz * gyyz + gupzz * gzzy);

  // :260-313 A~^ij and the Gamma-driver source without shift terms
  T Gamx_rhs, Gamy_rhs, Gamz_rhs;
  T Lapx, Lapy, Lapz;
  grad<T, F_LAP>(q, C, ord, Lapx, Lapy, Lapz);
  {
    T Kx, Ky, Kz;
    grad<T, F_TRK>(q, C, ord, Kx, Ky, Kz);
    if constexpr (Z4C) {  // Z4c_rhs.f90:582-586: K_,i + Theta_,i / 2
      T tx, ty, tz;
      grad<T, F_TZ>(q, C, ord, tx, ty, tz);
      Kx = Kx + tx / TWO;
      Ky = Ky + ty / TWO;
      Kz = Kz + tz / TWO;
    }
    const T Rxx = gupxx * gupxx * Axx + gupxy * gupxy * Ayy + gupxz * gupxz * Azz +
                  TWO * (gupxx * gupxy * Axy + gupxx * gupxz * Axz + gupxy * gupxz * Ayz);
    const T Ryy = gupxy * gupxy * Axx + gupyy * gupyy * Ayy + gupyz * gupyz * Azz +
                  TWO * (gupxy * gupyy * Axy + gupxy * gupyz * Axz + gupyy * gupyz * Ayz);
    const T Rzz = gupxz * gupxz * Axx + gupyz * gupyz * Ayy + gupzz * gupzz * Azz +
                  TWO * (gupxz * gupyz * Axy + gupxz * gupzz * Axz + gupyz * gupzz * Ayz);
    const T Rxy = gupxx * gupxy * Axx + gupxy * gupyy * Ayy + gupxz * gupyz * Azz +
                  (gupxx * gupyy + gupxy * gupxy) * Axy + (gupxx * gupyz + gupxz * gupxy) * Axz +
                  (gupxy * gupyz + gupxz * gupyy) * Ayz;
    const T Rxz = gupxx * gupxz * Axx + gupxy * gupyz * Ayy + gupxz * gupzz * Azz +
                  (gupxx * gupyz + gupxy * gupxz) * Axy + (gupxx * gupzz + gupxz * gupxz) * Axz +
                  (gupxy * gupzz + gupxz * gupyz) * Ayz;
    const T Ryz = gupxy * gupxz * Axx + gupyy * gupyz * Ayy + gupyz * gupzz * Azz +
                  (gupxy * gupyz + gupyy * gupxz) * Axy + (gupxy * gupzz + gupyz * gupxz) * Axz +
                  (gupyy * gupzz + gupyz * gupyz) * Ayz;
    Gamx_rhs = -TWO * (Lapx * Rxx + Lapy * Rxy + Lapz * Rxz) +
               TWO * alpn1 *
                   (-F3o2 / chin1 * (chix * Rxx + chiy * Rxy + chiz * Rxz) - gupxx * (F2o3 * Kx + EIGHT * PI * Sx) -
                    gupxy * (F2o3 * Ky + EIGHT * PI * Sy) - gupxz * (F2o3 * Kz + EIGHT * PI * Sz) + Gamxxx * Rxx +
                    Gamxyy * Ryy + Gamxzz * Rzz + TWO * (Gamxxy * Rxy + Gamxxz * Rxz + Gamxyz * Ryz));
    Gamy_rhs = -TWO * (Lapx * Rxy + Lapy * Ryy + Lapz * Ryz) +
               TWO * alpn1 *
                   (-F3o2 / chin1 * (chix * Rxy + chiy * Ryy + chiz * Ryz) - gupxy * (F2o3 * Kx + EIGHT * PI * Sx) -
                    gupyy * (F2o3 * Ky + EIGHT * PI * Sy) - gupyz * (F2o3 * Kz + EIGHT * PI * Sz) + Gamyxx * Rxx +
                    Gamyyy * Ryy + Gamyzz * Rzz + TWO * (Gamyxy * Rxy + Gamyxz * Rxz + Gamyyz * Ryz));
    Gamz_rhs = -TWO * (Lapx * Rxz + Lapy * Ryz + Lapz * Rzz) +
               TWO * alpn1 *
                   (-F3o2 / chin1 * (chix * Rxz + chiy * Ryz + chiz * Rzz) - gupxz * (F2o3 * Kx + EIGHT * PI * Sx) -
                    gupyz * (F2o3 * Ky + EIGHT * PI * Sy) - gupzz * (F2o3 * Kz + EIGHT * PI * Sz) + Gamzxx * Rxx +
                    Gamzyy * Ryy + Gamzzz * Rzz + TWO * (Gamzxy * Rxy + Gamzxz * Rxz + Gamzyz * Ryz));
  }

  // :315-353 shift second derivatives, Gam^i contraction, d Gam^i
  const T Gamxa = gupxx * Gamxxx + gupyy * Gamxyy + gupzz * Gamxzz +
                  TWO * (gupxy * Gamxxy + gupxz * Gamxxz + gupyz * Gamxyz);
  const T Gamya = gupxx * Gamyxx + gupyy * Gamyyy + gupzz * Gamyzz +
                  TWO * (gupxy * Gamyxy + gupxz * Gamyxz + gupyz * Gamyyz);
  const T Gamza = gupxx * Gamzxx + gupyy * Gamzyy + gupzz * Gamzzz +
                  TWO * (gupxy * Gamzxy + gupxz * Gamzxz + gupyz * Gamzyz);
  {
    T bx_xx, bx_xy, bx_xz, bx_yy, bx_yz, bx_zz;
    T by_xx, by_xy, by_xz, by_yy, by_yz, by_zz;
    T bz_xx, bz_xy, bz_xz, bz_yy, bz_yz, bz_zz;
    hess<T, F_BETAX>(q, C, ord, bx_xx, bx_xy, bx_xz, bx_yy, bx_yz, bx_zz);
    hess<T, F_BETAY>(q, C, ord, by_xx, by_xy, by_xz, by_yy, by_yz, by_zz);
    hess<T, F_BETAZ>(q, C, ord, bz_xx, bz_xy, bz_xz, bz_yy, bz_yz, bz_zz);
    const T fxx = bx_xx + by_xy + bz_xz;
    const T fxy = bx_xy + by_yy + bz_yz;
    const T fxz = bx_xz + by_yz + bz_zz;
    Gamx_rhs = Gamx_rhs + F2o3 * Gamxa * div_beta - Gamxa * betaxx - Gamya * betaxy - Gamza * betaxz +
               F1o3 * (gupxx * fxx + gupxy * fxy + gupxz * fxz) + gupxx * bx_xx + gupyy * bx_yy + gupzz * bx_zz +
               TWO * (gupxy * bx_xy + gupxz * bx_xz + gupyz * bx_yz);
    Gamy_rhs = Gamy_rhs + F2o3 * Gamya * div_beta - Gamxa * betayx - Gamya * betayy - Gamza * betayz +
               F1o3 * (gupxy * fxx + gupyy * fxy + gupyz * fxz) + gupxx * by_xx + gupyy * by_yy + gupzz * by_zz +
               TWO * (gupxy * by_xy + gupxz * by_xz + gupyz * by_yz);
    Gamz_rhs = Gamz_rhs + F2o3 * Gamza * div_beta - Gamxa * betazx - Gamya * betazy - Gamza * betazz +
               F1o3 * (gupxz * fxx + gupyz * fxy + gupzz * fxz) + gupxx * bz_xx + gupyy * bz_yy + gupzz * bz_zz +
               TWO * (gupxy * bz_xy + gupxz * bz_xz + gupyz * bz_yz);
  }
  // :797-799 (GAUGE 0) and the advection / dissipation of Gam^i and B^i
  if constexpr (Z4C) {
    // Z4c_rhs.f90:1231-1233 constraint damping (B^i takes the undamped source)
    finish_field<T, F_GAMX>(q, C, G, Gamx_rhs - TWO * alpn1 * kappa1 * (Gamx - Gamxa), betax, betay, betaz, ZEO, epi);
    finish_field<T, F_GAMY>(q, C, G, Gamy_rhs - TWO * alpn1 * kappa1 * (Gamy - Gamya), betax, betay, betaz, ZEO, epi);
    finish_field<T, F_GAMZ>(q, C, G, Gamz_rhs - TWO * alpn1 * kappa1 * (Gamz - Gamza), betax, betay, betaz, ZEO, epi);
  } else {
    finish_field<T, F_GAMX>(q, C, G, Gamx_rhs, betax, betay, betaz, ZEO, epi);
    finish_field<T, F_GAMY>(q, C, G, Gamy_rhs, betax, betay, betaz, ZEO, epi);
    finish_field<T, F_GAMZ>(q, C, G, Gamz_rhs, betax, betay, betaz, ZEO, epi);
  }
  finish_field<T, F_DTSFX>(q, C, G, Gamx_rhs - eta * dtSfx, betax, betay, betaz, ZEO, epi);
  finish_field<T, F_DTSFY>(q, C, G, Gamy_rhs - eta * dtSfy, betax, betay, betaz, ZEO, epi);
  finish_field<T, F_DTSFZ>(q, C, G, Gamz_rhs - eta * dtSfz, betax, betay, betaz, ZEO, epi);

  // :333-335 derivatives of Gam^i
  T Gamxx, Gamxy, Gamxz, Gamyx, Gamyy, Gamyz, Gamzx, Gamzy, Gamzz;
  grad<T, F_GAMX>(q, C, ord, Gamxx, Gamxy, Gamxz);
  grad<T, F_GAMY>(q, C, ord, Gamyx, Gamyy, Gamyz);
  grad<T, F_GAMZ>(q, C, ord, Gamzx, Gamzy, Gamzz);

  // :356-375 first kind of connection, stored in the gij_k names
  gxxx = gxx * Gamxxx + gxy * Gamyxx + gxz * Gamzxx;
  gxyx = gxx * Gamxxy + gxy * Gamyxy + gxz * Gamzxy;
  gxzx = gxx * Gamxxz + gxy * Gamyxz + gxz * Gamzxz;
  gyyx = gxx * Gamxyy + gxy * Gamyyy + gxz * Gamzyy;
  gyzx = gxx * Gamxyz + gxy * Gamyyz + gxz * Gamzyz;
  gzzx = gxx * Gamxzz + gxy * Gamyzz + gxz * Gamzzz;
  gxxy = gxy * Gamxxx + gyy * Gamyxx + gyz * Gamzxx;
  gxyy = gxy * Gamxxy + gyy * Gamyxy + gyz * Gamzxy;
  gxzy = gxy * Gamxxz + gyy * Gamyxz + gyz * Gamzxz;
  gyyy = gxy * Gamxyy + gyy * Gamyyy + gyz * Gamzyy;
  gyzy = gxy * Gamxyz + gyy * Gamyyz + gyz * Gamzyz;
  gzzy = gxy * Gamxzz + gyy * Gamyzz + gyz * Gamzzz;
  gxxz = gxz * Gamxxx + gyz * Gamyxx + gzz * Gamzxx;
  gxyz = gxz * Gamxxy + gyz * Gamyxy + gzz * Gamzxy;
  gxzz = gxz * Gamxxz + gyz * Gamyxz + gzz * Gamzxz;
  gyyz = gxz * Gamxyy + gyz * Gamyyy + gzz * Gamzyy;
  gyzz = gxz * Gamxyz + gyz * Gamyyz + gzz * Gamzyz;
  gzzz = gxz * Gamxzz + gyz * Gamyzz + gzz * Gamzzz;

  // :378-400 gup^kl d_k d_l g_ij, one metric component at a time
  T Rxx, Ryy, Rzz, Rxy, Rxz, Ryz;
  {
    T fxx, fxy, fxz, fyy, fyz, fzz;
#define AMSS_RC(F, R)                                                                      \
    hess<T, F>(q, C, ord, fxx, fxy, fxz, fyy, fyz, fzz);                                   \
    R = gupxx * fxx + gupyy * fyy + gupzz * fzz + (gupxy * fxy + gupxz * fxz + gupyz * fyz) * TWO;
    AMSS_RC(F_GXX, Rxx)
    AMSS_RC(F_GYY, Ryy)
    AMSS_RC(F_GZZ, Rzz)
    AMSS_RC(F_GXY, Rxy)
    AMSS_RC(F_GXZ, Rxz)
    AMSS_RC(F_GYZ, Ryz)
#undef AMSS_RC
  }
  {
    // :402-601 conformal Ricci tensor
    const T Rxx_r = -HALF * Rxx +
      gxx * Gamxx + gxy * Gamyx + gxz * Gamzx +
      Gamxa * gxxx + Gamya * gxyx + Gamza * gxzx +
      gupxx * (TWO * (Gamxxx * gxxx + Gamyxx * gxyx + Gamzxx * gxzx) +
      Gamxxx * gxxx + Gamyxx * gxxy + Gamzxx * gxxz) +
      gupxy * (TWO * (Gamxxx * gxyx + Gamyxx * gyyx + Gamzxx * gyzx +
      Gamxxy * gxxx + Gamyxy * gxyx + Gamzxy * gxzx) +
      Gamxxy * gxxx + Gamyxy * gxxy + Gamzxy * gxxz +
      Gamxxx * gxyx + Gamyxx * gxyy + Gamzxx * gxyz) +
      gupxz * (TWO * (Gamxxx * gxzx + Gamyxx * gyzx + Gamzxx * gzzx +
      Gamxxz * gxxx + Gamyxz * gxyx + Gamzxz * gxzx) +
      Gamxxz * gxxx + Gamyxz * gxxy + Gamzxz * gxxz +
      Gamxxx * gxzx + Gamyxx * gxzy + Gamzxx * gxzz) +
      gupyy * (TWO * (Gamxxy * gxyx + Gamyxy * gyyx + Gamzxy * gyzx) +
      Gamxxy * gxyx + Gamyxy * gxyy + Gamzxy * gxyz) +
      gupyz * (TWO * (Gamxxy * gxzx + Gamyxy * gyzx + Gamzxy * gzzx +
      Gamxxz * gxyx + Gamyxz * gyyx + Gamzxz * gyzx) +
      Gamxxz * gxyx + Gamyxz * gxyy + Gamzxz * gxyz +
      Gamxxy * gxzx + Gamyxy * gxzy + Gamzxy * gxzz) +
      gupzz * (TWO * (Gamxxz * gxzx + Gamyxz * gyzx + Gamzxz * gzzx) +
      Gamxxz * gxzx + Gamyxz * gxzy + Gamzxz * gxzz);
    const T Ryy_r = -HALF * Ryy +
      gxy * Gamxy + gyy * Gamyy + gyz * Gamzy +
      Gamxa * gxyy + Gamya * gyyy + Gamza * gyzy +
      gupxx * (TWO * (Gamxxy * gxxy + Gamyxy * gxyy + Gamzxy * gxzy) +
      Gamxxy * gxyx + Gamyxy * gxyy + Gamzxy * gxyz) +
      gupxy * (TWO * (Gamxxy * gxyy + Gamyxy * gyyy + Gamzxy * gyzy +
      Gamxyy * gxxy + Gamyyy * gxyy + Gamzyy * gxzy) +
      Gamxyy * gxyx + Gamyyy * gxyy + Gamzyy * gxyz +
      Gamxxy * gyyx + Gamyxy * gyyy + Gamzxy * gyyz) +
      gupxz * (TWO * (Gamxxy * gxzy + Gamyxy * gyzy + Gamzxy * gzzy +
      Gamxyz * gxxy + Gamyyz * gxyy + Gamzyz * gxzy) +
      Gamxyz * gxyx + Gamyyz * gxyy + Gamzyz * gxyz +
      Gamxxy * gyzx + Gamyxy * gyzy + Gamzxy * gyzz) +
      gupyy * (TWO * (Gamxyy * gxyy + Gamyyy * gyyy + Gamzyy * gyzy) +
      Gamxyy * gyyx + Gamyyy * gyyy + Gamzyy * gyyz) +
      gupyz * (TWO * (Gamxyy * gxzy + Gamyyy * gyzy + Gamzyy * gzzy +
      Gamxyz * gxyy + Gamyyz * gyyy + Gamzyz * gyzy) +
      Gamxyz * gyyx + Gamyyz * gyyy + Gamzyz * gyyz +
      Gamxyy * gyzx + Gamyyy * gyzy + Gamzyy * gyzz) +
      gupzz * (TWO * (Gamxyz * gxzy + Gamyyz * gyzy + Gamzyz * gzzy) +
      Gamxyz * gyzx + Gamyyz * gyzy + Gamzyz * gyzz);
    const T Rzz_r = -HALF * Rzz +
      gxz * Gamxz + gyz * Gamyz + gzz * Gamzz +
      Gamxa * gxzz + Gamya * gyzz + Gamza * gzzz +
      gupxx * (TWO * (Gamxxz * gxxz + Gamyxz * gxyz + Gamzxz * gxzz) +
      Gamxxz * gxzx + Gamyxz * gxzy + Gamzxz * gxzz) +
      gupxy * (TWO * (Gamxxz * gxyz + Gamyxz * gyyz + Gamzxz * gyzz +
      Gamxyz * gxxz + Gamyyz * gxyz + Gamzyz * gxzz) +
      Gamxyz * gxzx + Gamyyz * gxzy + Gamzyz * gxzz +
      Gamxxz * gyzx + Gamyxz * gyzy + Gamzxz * gyzz) +
      gupxz * (TWO * (Gamxxz * gxzz + Gamyxz * gyzz + Gamzxz * gzzz +
      Gamxzz * gxxz + Gamyzz * gxyz + Gamzzz * gxzz) +
      Gamxzz * gxzx + Gamyzz * gxzy + Gamzzz * gxzz +
      Gamxxz * gzzx + Gamyxz * gzzy + Gamzxz * gzzz) +
      gupyy * (TWO * (Gamxyz * gxyz + Gamyyz * gyyz + Gamzyz * gyzz) +
      Gamxyz * gyzx + Gamyyz * gyzy + Gamzyz * gyzz) +
      gupyz * (TWO * (Gamxyz * gxzz + Gamyyz * gyzz + Gamzyz * gzzz +
      Gamxzz * gxyz + Gamyzz * gyyz + Gamzzz * gyzz) +
      Gamxzz * gyzx + Gamyzz * gyzy + Gamzzz * gyzz +
      Gamxyz * gzzx + Gamyyz * gzzy + Gamzyz * gzzz) +
      gupzz * (TWO * (Gamxzz * gxzz + Gamyzz * gyzz + Gamzzz * gzzz) +
      Gamxzz * gzzx + Gamyzz * gzzy + Gamzzz * gzzz);
    const T Rxy_r = HALF * (-Rxy +
      gxx * Gamxy + gxy * Gamyy + gxz * Gamzy +
      gxy * Gamxx + gyy * Gamyx + gyz * Gamzx +
      Gamxa * gxyx + Gamya * gyyx + Gamza * gyzx +
      Gamxa * gxxy + Gamya * gxyy + Gamza * gxzy) +
      gupxx * (Gamxxx * gxxy + Gamyxx * gxyy + Gamzxx * gxzy +
      Gamxxy * gxxx + Gamyxy * gxyx + Gamzxy * gxzx +
      Gamxxx * gxyx + Gamyxx * gxyy + Gamzxx * gxyz) +
      gupxy * (Gamxxx * gxyy + Gamyxx * gyyy + Gamzxx * gyzy +
      Gamxxy * gxyx + Gamyxy * gyyx + Gamzxy * gyzx +
      Gamxxy * gxyx + Gamyxy * gxyy + Gamzxy * gxyz +
      Gamxxy * gxxy + Gamyxy * gxyy + Gamzxy * gxzy +
      Gamxyy * gxxx + Gamyyy * gxyx + Gamzyy * gxzx +
      Gamxxx * gyyx + Gamyxx * gyyy + Gamzxx * gyyz) +
      gupxz * (Gamxxx * gxzy + Gamyxx * gyzy + Gamzxx * gzzy +
      Gamxxy * gxzx + Gamyxy * gyzx + Gamzxy * gzzx +
      Gamxxz * gxyx + Gamyxz * gxyy + Gamzxz * gxyz +
      Gamxxz * gxxy + Gamyxz * gxyy + Gamzxz * gxzy +
      Gamxyz * gxxx + Gamyyz * gxyx + Gamzyz * gxzx +
      Gamxxx * gyzx + Gamyxx * gyzy + Gamzxx * gyzz) +
      gupyy * (Gamxxy * gxyy + Gamyxy * gyyy + Gamzxy * gyzy +
      Gamxyy * gxyx + Gamyyy * gyyx + Gamzyy * gyzx +
      Gamxxy * gyyx + Gamyxy * gyyy + Gamzxy * gyyz) +
      gupyz * (Gamxxy * gxzy + Gamyxy * gyzy + Gamzxy * gzzy +
      Gamxyy * gxzx + Gamyyy * gyzx + Gamzyy * gzzx +
      Gamxxz * gyyx + Gamyxz * gyyy + Gamzxz * gyyz +
      Gamxxz * gxyy + Gamyxz * gyyy + Gamzxz * gyzy +
      Gamxyz * gxyx + Gamyyz * gyyx + Gamzyz * gyzx +
      Gamxxy * gyzx + Gamyxy * gyzy + Gamzxy * gyzz) +
      gupzz * (Gamxxz * gxzy + Gamyxz * gyzy + Gamzxz * gzzy +
      Gamxyz * gxzx + Gamyyz * gyzx + Gamzyz * gzzx +
      Gamxxz * gyzx + Gamyxz * gyzy + Gamzxz * gyzz);
    const T Rxz_r = HALF * (-Rxz +
      gxx * Gamxz + gxy * Gamyz + gxz * Gamzz +
      gxz * Gamxx + gyz * Gamyx + gzz * Gamzx +
      Gamxa * gxzx + Gamya * gyzx + Gamza * gzzx +
      Gamxa * gxxz + Gamya * gxyz + Gamza * gxzz) +
      gupxx * (Gamxxx * gxxz + Gamyxx * gxyz + Gamzxx * gxzz +
      Gamxxz * gxxx + Gamyxz * gxyx + Gamzxz * gxzx +
      Gamxxx * gxzx + Gamyxx * gxzy + Gamzxx * gxzz) +
      gupxy * (Gamxxx * gxyz + Gamyxx * gyyz + Gamzxx * gyzz +
      Gamxxz * gxyx + Gamyxz * gyyx + Gamzxz * gyzx +
      Gamxxy * gxzx + Gamyxy * gxzy + Gamzxy * gxzz +
      Gamxxy * gxxz + Gamyxy * gxyz + Gamzxy * gxzz +
      Gamxyz * gxxx + Gamyyz * gxyx + Gamzyz * gxzx +
      Gamxxx * gyzx + Gamyxx * gyzy + Gamzxx * gyzz) +
      gupxz * (Gamxxx * gxzz + Gamyxx * gyzz + Gamzxx * gzzz +
      Gamxxz * gxzx + Gamyxz * gyzx + Gamzxz * gzzx +
      Gamxxz * gxzx + Gamyxz * gxzy + Gamzxz * gxzz +
      Gamxxz * gxxz + Gamyxz * gxyz + Gamzxz * gxzz +
      Gamxzz * gxxx + Gamyzz * gxyx + Gamzzz * gxzx +
      Gamxxx * gzzx + Gamyxx * gzzy + Gamzxx * gzzz) +
      gupyy * (Gamxxy * gxyz + Gamyxy * gyyz + Gamzxy * gyzz +
      Gamxyz * gxyx + Gamyyz * gyyx + Gamzyz * gyzx +
      Gamxxy * gyzx + Gamyxy * gyzy + Gamzxy * gyzz) +
      gupyz * (Gamxxy * gxzz + Gamyxy * gyzz + Gamzxy * gzzz +
      Gamxyz * gxzx + Gamyyz * gyzx + Gamzyz * gzzx +
      Gamxxz * gyzx + Gamyxz * gyzy + Gamzxz * gyzz +
      Gamxxz * gxyz + Gamyxz * gyyz + Gamzxz * gyzz +
      Gamxzz * gxyx + Gamyzz * gyyx + Gamzzz * gyzx +
      Gamxxy * gzzx + Gamyxy * gzzy + Gamzxy * gzzz) +
      gupzz * (Gamxxz * gxzz + Gamyxz * gyzz + Gamzxz * gzzz +
      Gamxzz * gxzx + Gamyzz * gyzx + Gamzzz * gzzx +
      Gamxxz * gzzx + Gamyxz * gzzy + Gamzxz * gzzz);
    const T Ryz_r = HALF * (-Ryz +
      gxy * Gamxz + gyy * Gamyz + gyz * Gamzz +
      gxz * Gamxy + gyz * Gamyy + gzz * Gamzy +
      Gamxa * gxzy + Gamya * gyzy + Gamza * gzzy +
      Gamxa * gxyz + Gamya * gyyz + Gamza * gyzz) +
      gupxx * (Gamxxy * gxxz + Gamyxy * gxyz + Gamzxy * gxzz +
      Gamxxz * gxxy + Gamyxz * gxyy + Gamzxz * gxzy +
      Gamxxy * gxzx + Gamyxy * gxzy + Gamzxy * gxzz) +
      gupxy * (Gamxxy * gxyz + Gamyxy * gyyz + Gamzxy * gyzz +
      Gamxxz * gxyy + Gamyxz * gyyy + Gamzxz * gyzy +
      Gamxyy * gxzx + Gamyyy * gxzy + Gamzyy * gxzz +
      Gamxyy * gxxz + Gamyyy * gxyz + Gamzyy * gxzz +
      Gamxyz * gxxy + Gamyyz * gxyy + Gamzyz * gxzy +
      Gamxxy * gyzx + Gamyxy * gyzy + Gamzxy * gyzz) +
      gupxz * (Gamxxy * gxzz + Gamyxy * gyzz + Gamzxy * gzzz +
      Gamxxz * gxzy + Gamyxz * gyzy + Gamzxz * gzzy +
      Gamxyz * gxzx + Gamyyz * gxzy + Gamzyz * gxzz +
      Gamxyz * gxxz + Gamyyz * gxyz + Gamzyz * gxzz +
      Gamxzz * gxxy + Gamyzz * gxyy + Gamzzz * gxzy +
      Gamxxy * gzzx + Gamyxy * gzzy + Gamzxy * gzzz) +
      gupyy * (Gamxyy * gxyz + Gamyyy * gyyz + Gamzyy * gyzz +
      Gamxyz * gxyy + Gamyyz * gyyy + Gamzyz * gyzy +
      Gamxyy * gyzx + Gamyyy * gyzy + Gamzyy * gyzz) +
      gupyz * (Gamxyy * gxzz + Gamyyy * gyzz + Gamzyy * gzzz +
      Gamxyz * gxzy + Gamyyz * gyzy + Gamzyz * gzzy +
      Gamxyz * gyzx + Gamyyz * gyzy + Gamzyz * gyzz +
      Gamxyz * gxyz + Gamyyz * gyyz + Gamzyz * gyzz +
      Gamxzz * gxyy + Gamyzz * gyyy + Gamzzz * gyzy +
      Gamxyy * gzzx + Gamyyy * gzzy + Gamzyy * gzzz) +
      gupzz * (Gamxyz * gxzz + Gamyyz * gyzz + Gamzyz * gzzz +
      Gamxzz * gxzy + Gamyzz * gyzy + Gamzzz * gzzy +
      Gamxyz * gzzx + Gamyyz * gzzy + Gamzyz * gzzz);
    Rxx = Rxx_r; Ryy = Ryy_r; Rzz = Rzz_r; Rxy = Rxy_r; Rxz = Rxz_r; Ryz = Ryz_r;
  }

  // :603-626 chi part of the Ricci tensor
  T fxx, fxy, fxz, fyy, fyz, fzz;
  hess<T, F_CHI>(q, C, ord, fxx, fxy, fxz, fyy, fyz, fzz);
  fxx = fxx - Gamxxx * chix - Gamyxx * chiy - Gamzxx * chiz;
  fxy = fxy - Gamxxy * chix - Gamyxy * chiy - Gamzxy * chiz;
  fxz = fxz - Gamxxz * chix - Gamyxz * chiy - Gamzxz * chiz;
  fyy = fyy - Gamxyy * chix - Gamyyy * chiy - Gamzyy * chiz;
  fyz = fyz - Gamxyz * chix - Gamyyz * chiy - Gamzyz * chiz;
  fzz = fzz - Gamxzz * chix - Gamyzz * chiy - Gamzzz * chiz;
  {
    const T f = gupxx * (fxx - F3o2 / chin1 * chix * chix) + gupyy * (fyy - F3o2 / chin1 * chiy * chiy) +
                gupzz * (fzz - F3o2 / chin1 * chiz * chiz) + TWO * gupxy * (fxy - F3o2 / chin1 * chix * chiy) +
                TWO * gupxz * (fxz - F3o2 / chin1 * chix * chiz) + TWO * gupyz * (fyz - F3o2 / chin1 * chiy * chiz);
    Rxx = Rxx + (fxx - chix * chix / chin1 / TWO + gxx * f) / chin1 / TWO;
    Ryy = Ryy + (fyy - chiy * chiy / chin1 / TWO + gyy * f) / chin1 / TWO;
    Rzz = Rzz + (fzz - chiz * chiz / chin1 / TWO + gzz * f) / chin1 / TWO;
    Rxy = Rxy + (fxy - chix * chiy / chin1 / TWO + gxy * f) / chin1 / TWO;
    Rxz = Rxz + (fxz - chix * chiz / chin1 / TWO + gxz * f) / chin1 / TWO;
    Ryz = Ryz + (fyz - chiy * chiz / chin1 / TWO + gyz * f) / chin1 / TWO;
  }
  // Z4c_rhs.f90:913-915: R / chi, the trace of the A~_ij source and of H
  T Hc = ZEO;
  if constexpr (Z4C) Hc = gupxx * Rxx + gupyy * Ryy + gupzz * Rzz + TWO * (gupxy * Rxy + gupxz * Rxz + gupyz * Ryz);

  // :629-660 D_i D_j alpha with the physical connection
  hess<T, F_LAP>(q, C, ord, fxx, fxy, fxz, fyy, fyz, fzz);
  {
    const T cx = (gupxx * chix + gupxy * chiy + gupxz * chiz) / chin1;
    const T cy = (gupxy * chix + gupyy * chiy + gupyz * chiz) / chin1;
    const T cz = (gupxz * chix + gupyz * chiy + gupzz * chiz) / chin1;
    Gamxxx = Gamxxx - ((chix + chix) / chin1 - gxx * cx) * HALF;
    Gamyxx = Gamyxx - (-gxx * cy) * HALF;
    Gamzxx = Gamzxx - (-gxx * cz) * HALF;
    Gamxyy = Gamxyy - (-gyy * cx) * HALF;
    Gamyyy = Gamyyy - ((chiy + chiy) / chin1 - gyy * cy) * HALF;
    Gamzyy = Gamzyy - (-gyy * cz) * HALF;
    Gamxzz = Gamxzz - (-gzz * cx) * HALF;
    Gamyzz = Gamyzz - (-gzz * cy) * HALF;
    Gamzzz = Gamzzz - ((chiz + chiz) / chin1 - gzz * cz) * HALF;
    Gamxxy = Gamxxy - (chiy / chin1 - gxy * cx) * HALF;
    Gamyxy = Gamyxy - (chix / chin1 - gxy * cy) * HALF;
    Gamzxy = Gamzxy - (-gxy * cz) * HALF;
    Gamxxz = Gamxxz - (chiz / chin1 - gxz * cx) * HALF;
    Gamyxz = Gamyxz - (-gxz * cy) * HALF;
    Gamzxz = Gamzxz - (chix / chin1 - gxz * cz) * HALF;
    Gamxyz = Gamxyz - (-gyz * cx) * HALF;
    Gamyyz = Gamyyz - (chiz / chin1 - gyz * cy) * HALF;
    Gamzyz = Gamzyz - (chiy / chin1 - gyz * cz) * HALF;
  }
  fxx = fxx - Gamxxx * Lapx - Gamyxx * Lapy - Gamzxx * Lapz;
  fyy = fyy - Gamxyy * Lapx - Gamyyy * Lapy - Gamzyy * Lapz;
  fzz = fzz - Gamxzz * Lapx - Gamyzz * Lapy - Gamzzz * Lapz;
  fxy = fxy - Gamxxy * Lapx - Gamyxy * Lapy - Gamzxy * Lapz;
  fxz = fxz - Gamxxz * Lapx - Gamyxz * Lapy - Gamzxz * Lapz;
  fyz = fyz - Gamxyz * Lapx - Gamyyz * Lapy - Gamzyz * Lapz;

  // :663-787 trK and A~_ij
  T trK_rhs = gupxx * fxx + gupyy * fyy + gupzz * fzz + TWO * (gupxy * fxy + gupxz * fxz + gupyz * fyz);
  // A~_il A~^l_j and its trace pieces, :729-746 (the same sums enter :669-694)
  const T AAxx = gupxx * Axx * Axx + gupyy * Axy * Axy + gupzz * Axz * Axz +
                 TWO * (gupxy * Axx * Axy + gupxz * Axx * Axz + gupyz * Axy * Axz);
  const T AAyy = gupxx * Axy * Axy + gupyy * Ayy * Ayy + gupzz * Ayz * Ayz +
                 TWO * (gupxy * Axy * Ayy + gupxz * Axy * Ayz + gupyz * Ayy * Ayz);
  const T AAzz = gupxx * Axz * Axz + gupyy * Ayz * Ayz + gupzz * Azz * Azz +
                 TWO * (gupxy * Axz * Ayz + gupxz * Axz * Azz + gupyz * Ayz * Azz);
  const T AAxy = gupxx * Axx * Axy + gupyy * Axy * Ayy + gupzz * Axz * Ayz + gupxy * (Axx * Ayy + Axy * Axy) +
                 gupxz * (Axx * Ayz + Axz * Axy) + gupyz * (Axy * Ayz + Axz * Ayy);
  const T AAxz = gupxx * Axx * Axz + gupyy * Axy * Ayz + gupzz * Axz * Azz + gupxy * (Axx * Ayz + Axy * Axz) +
                 gupxz * (Axx * Azz + Axz * Axz) + gupyz * (Axy * Azz + Axz * Ayz);
  const T AAyz = gupxx * Axy * Axz + gupyy * Ayy * Ayz + gupzz * Ayz * Azz + gupxy * (Axy * Ayz + Ayy * Axz) +
                 gupxz * (Axy * Azz + Ayz * Axz) + gupyz * (Ayy * Azz + Ayz * Ayz);
  // A_ij A^ij as written at :670-694 (sum of gup^ij times the rows above)
  const T AijAij = gupxx * AAxx + gupyy * AAyy + gupzz * AAzz + TWO * (gupxy * AAxy + gupxz * AAxz + gupyz * AAyz);
  {
    T S, f, axx, axy, axz, ayy, ayz, azz;
    if constexpr (Z4C) {
      // Z4c_rhs.f90:964-982: the trace of the source from the Ricci scalar
      const T sxx = EIGHT * PI * alpn1 * Sxx + fxx, sxy = EIGHT * PI * alpn1 * Sxy + fxy;
      const T sxz = EIGHT * PI * alpn1 * Sxz + fxz, syy = EIGHT * PI * alpn1 * Syy + fyy;
      const T syz = EIGHT * PI * alpn1 * Syz + fyz, szz = EIGHT * PI * alpn1 * Szz + fzz;
      f = gupxx * sxx + gupyy * syy + gupzz * szz + TWO * (gupxy * sxy + gupxz * sxz + gupyz * syz);
      f = F1o3 * (Hc * alpn1 - f);
      axx = alpn1 * Rxx - sxx; axy = alpn1 * Rxy - sxy; axz = alpn1 * Rxz - sxz;
      ayy = alpn1 * Ryy - syy; ayz = alpn1 * Ryz - syz; azz = alpn1 * Rzz - szz;
    } else {
      S = chin1 * (gupxx * Sxx + gupyy * Syy + gupzz * Szz + TWO * (gupxy * Sxy + gupxz * Sxz + gupyz * Syz));
      f = F2o3 * trK * trK - AijAij - T(16) * PI * rho + EIGHT * PI * S;
      f = -F1o3 * (gupxx * fxx + gupyy * fyy + gupzz * fzz + TWO * (gupxy * fxy + gupxz * fxz + gupyz * fyz) +
                   alpn1 / chin1 * f);
      axx = alpn1 * (Rxx - EIGHT * PI * Sxx) - fxx;
      axy = alpn1 * (Rxy - EIGHT * PI * Sxy) - fxy;
      axz = alpn1 * (Rxz - EIGHT * PI * Sxz) - fxz;
      ayy = alpn1 * (Ryy - EIGHT * PI * Syy) - fyy;
      ayz = alpn1 * (Ryz - EIGHT * PI * Syz) - fyz;
      azz = alpn1 * (Rzz - EIGHT * PI * Szz) - fzz;
    }
    T Axx_rhs = axx - gxx * f, Ayy_rhs = ayy - gyy * f, Azz_rhs = azz - gzz * f;
    T Axy_rhs = axy - gxy * f, Axz_rhs = axz - gxz * f, Ayz_rhs = ayz - gyz * f;
    const T fc = chin1;
    trK_rhs = fc * trK_rhs;
    Axx_rhs = fc * Axx_rhs + alpn1 * (trKd * Axx - TWO * AAxx) + TWO * (Axx * betaxx + Axy * betayx + Axz * betazx) -
              F2o3 * Axx * div_beta;
    Ayy_rhs = fc * Ayy_rhs + alpn1 * (trKd * Ayy - TWO * AAyy) + TWO * (Axy * betaxy + Ayy * betayy + Ayz * betazy) -
              F2o3 * Ayy * div_beta;
    Azz_rhs = fc * Azz_rhs + alpn1 * (trKd * Azz - TWO * AAzz) + TWO * (Axz * betaxz + Ayz * betayz + Azz * betazz) -
              F2o3 * Azz * div_beta;
    Axy_rhs = fc * Axy_rhs + alpn1 * (trKd * Axy - TWO * AAxy) + Axx * betaxy + Axz * betazy + Ayy * betayx +
              Ayz * betazx + F1o3 * Axy * div_beta - Axy * betazz;
    Ayz_rhs = fc * Ayz_rhs + alpn1 * (trKd * Ayz - TWO * AAyz) + Axy * betaxz + Ayy * betayz + Axz * betaxy +
              Azz * betazy + F1o3 * Ayz * div_beta - Ayz * betaxx;
    Axz_rhs = fc * Axz_rhs + alpn1 * (trKd * Axz - TWO * AAxz) + Axx * betaxz + Axy * betayz + Ayz * betayx +
              Azz * betazx + F1o3 * Axz * div_beta - Axz * betayy;
    S = fc * (gupxx * Sxx + gupyy * Syy + gupzz * Szz + TWO * (gupxy * Sxy + gupxz * Sxz + gupyz * Syz));
    trK_rhs = -trK_rhs + alpn1 * (F1o3 * trKd * trKd + gupxx * AAxx + gupyy * AAyy + gupzz * AAzz +
                                  TWO * (gupxy * AAxy + gupxz * AAxz + gupyz * AAyz) + FOUR * PI * (rho + S));
    finish_field<T, F_AXX>(q, C, G, Axx_rhs, betax, betay, betaz, ZEO, epi);
    finish_field<T, F_AXY>(q, C, G, Axy_rhs, betax, betay, betaz, ZEO, epi);
    finish_field<T, F_AXZ>(q, C, G, Axz_rhs, betax, betay, betaz, ZEO, epi);
    finish_field<T, F_AYY>(q, C, G, Ayy_rhs, betax, betay, betaz, ZEO, epi);
    finish_field<T, F_AYZ>(q, C, G, Ayz_rhs, betax, betay, betaz, ZEO, epi);
    finish_field<T, F_AZZ>(q, C, G, Azz_rhs, betax, betay, betaz, ZEO, epi);
    if constexpr (Z4C) {
      // Z4c_rhs.f90:1230 damping; :1077-1110, :1165, :1229 Theta
      finish_field<T, F_TRK>(q, C, G, trK_rhs + alpn1 * kappa1 * (ONE - kappa2) * TZ, betax, betay, betaz, ZEO, epi);
      const T Hcon = chin1 * Hc + F2o3 * trKd * trKd - AijAij - T(16) * PI * rho;
      finish_field<T, F_TZ>(q, C, G, alpn1 * Hcon / TWO - alpn1 * (TWO + kappa2) * kappa1 * TZ, betax, betay, betaz,
                            ZEO, epi);
    } else {
      finish_field<T, F_TRK>(q, C, G, trK_rhs, betax, betay, betaz, ZEO, epi);
    }
  }

  // Hamiltonian constraint (bssn_rhs.f90:1047-1075, the BSSN form that
  // constraint_bssn also evaluates) for epilogues that ask for it: the
  // adjoint generator records it as the integrand of its loss.
  if constexpr (epi_wants_ham<E>::value) {
    const T h = gupxx * Rxx + gupyy * Ryy + gupzz * Rzz + TWO * (gupxy * Rxy + gupxz * Rxz + gupyz * Ryz);
    epi.ham(chin1 * h + F2o3 * trK * trK - AijAij - T(16) * PI * rho);
  }

  if constexpr (AUX) {
    const long long s = aux.fs;
    if (aux.gamma) {   // the constraint monitor asks for the residuals only
      double* gm = aux.gamma + q.p;
      gm[0] = Gamxxx; gm[s] = Gamxxy; gm[2 * s] = Gamxxz; gm[3 * s] = Gamxyy; gm[4 * s] = Gamxyz; gm[5 * s] = Gamxzz;
      gm[6 * s] = Gamyxx; gm[7 * s] = Gamyxy; gm[8 * s] = Gamyxz; gm[9 * s] = Gamyyy; gm[10 * s] = Gamyyz;
      gm[11 * s] = Gamyzz; gm[12 * s] = Gamzxx; gm[13 * s] = Gamzxy; gm[14 * s] = Gamzxz; gm[15 * s] = Gamzyy;
      gm[16 * s] = Gamzyz; gm[17 * s] = Gamzzz;
    }
    if (aux.ricci) {
      double* rc = aux.ricci + q.p;
      rc[0] = Rxx; rc[s] = Rxy; rc[2 * s] = Rxz; rc[3 * s] = Ryy; rc[4 * s] = Ryz; rc[5 * s] = Rzz;
    }
    if (aux.co == 0) {
      // :1047-1075 Hamiltonian constraint
      double* o = aux.cons + q.p;
      T h = gupxx * Rxx + gupyy * Ryy + gupzz * Rzz + TWO * (gupxy * Rxy + gupxz * Rxz + gupyz * Ryz);
      o[0] = chin1 * h + F2o3 * trK * trK - AijAij - T(16) * PI * rho;
      // :1079-1134 momentum constraint
      T axxx, axxy, axxz, axyx, axyy, axyz, axzx, axzy, axzz, ayyx, ayyy, ayyz, ayzx, ayzy, ayzz, azzx, azzy, azzz;
      const PointGates& g = G;
      grad<T, F_AXX>(q, C, g.ord, axxx, axxy, axxz);
      grad<T, F_AXY>(q, C, g.ord, axyx, axyy, axyz);
      grad<T, F_AXZ>(q, C, g.ord, axzx, axzy, axzz);
      grad<T, F_AYY>(q, C, g.ord, ayyx, ayyy, ayyz);
      grad<T, F_AYZ>(q, C, g.ord, ayzx, ayzy, ayzz);
      grad<T, F_AZZ>(q, C, g.ord, azzx, azzy, azzz);
      axxx = axxx - (Gamxxx * Axx + Gamyxx * Axy + Gamzxx * Axz + Gamxxx * Axx + Gamyxx * Axy + Gamzxx * Axz) - chix * Axx / chin1;
      axyx = axyx - (Gamxxy * Axx + Gamyxy * Axy + Gamzxy * Axz + Gamxxx * Axy + Gamyxx * Ayy + Gamzxx * Ayz) - chix * Axy / chin1;
      axzx = axzx - (Gamxxz * Axx + Gamyxz * Axy + Gamzxz * Axz + Gamxxx * Axz + Gamyxx * Ayz + Gamzxx * Azz) - chix * Axz / chin1;
      ayyx = ayyx - (Gamxxy * Axy + Gamyxy * Ayy + Gamzxy * Ayz + Gamxxy * Axy + Gamyxy * Ayy + Gamzxy * Ayz) - chix * Ayy / chin1;
      ayzx = ayzx - (Gamxxz * Axy + Gamyxz * Ayy + Gamzxz * Ayz + Gamxxy * Axz + Gamyxy * Ayz + Gamzxy * Azz) - chix * Ayz / chin1;
      azzx = azzx - (Gamxxz * Axz + Gamyxz * Ayz + Gamzxz * Azz + Gamxxz * Axz + Gamyxz * Ayz + Gamzxz * Azz) - chix * Azz / chin1;
      axxy = axxy - (Gamxxy * Axx + Gamyxy * Axy + Gamzxy * Axz + Gamxxy * Axx + Gamyxy * Axy + Gamzxy * Axz) - chiy * Axx / chin1;
      axyy = axyy - (Gamxyy * Axx + Gamyyy * Axy + Gamzyy * Axz + Gamxxy * Axy + Gamyxy * Ayy + Gamzxy * Ayz) - chiy * Axy / chin1;
      axzy = axzy - (Gamxyz * Axx + Gamyyz * Axy + Gamzyz * Axz + Gamxxy * Axz + Gamyxy * Ayz + Gamzxy * Azz) - chiy * Axz / chin1;
      ayyy = ayyy - (Gamxyy * Axy + Gamyyy * Ayy + Gamzyy * Ayz + Gamxyy * Axy + Gamyyy * Ayy + Gamzyy * Ayz) - chiy * Ayy / chin1;
      ayzy = ayzy - (Gamxyz * Axy + Gamyyz * Ayy + Gamzyz * Ayz + Gamxyy * Axz + Gamyyy * Ayz + Gamzyy * Azz) - chiy * Ayz / chin1;
      azzy = azzy - (Gamxyz * Axz + Gamyyz * Ayz + Gamzyz * Azz + Gamxyz * Axz + Gamyyz * Ayz + Gamzyz * Azz) - chiy * Azz / chin1;
      axxz = axxz - (Gamxxz * Axx + Gamyxz * Axy + Gamzxz * Axz + Gamxxz * Axx + Gamyxz * Axy + Gamzxz * Axz) - chiz * Axx / chin1;
      axyz = axyz - (Gamxyz * Axx + Gamyyz * Axy + Gamzyz * Axz + Gamxxz * Axy + Gamyxz * Ayy + Gamzxz * Ayz) - chiz * Axy / chin1;
      axzz = axzz - (Gamxzz * Axx + Gamyzz * Axy + Gamzzz * Axz + Gamxxz * Axz + Gamyxz * Ayz + Gamzxz * Azz) - chiz * Axz / chin1;
      ayyz = ayyz - (Gamxyz * Axy + Gamyyz * Ayy + Gamzyz * Ayz + Gamxyz * Axy + Gamyyz * Ayy + Gamzyz * Ayz) - chiz * Ayy / chin1;
      ayzz = ayzz - (Gamxzz * Axy + Gamyzz * Ayy + Gamzzz * Ayz + Gamxyz * Axz + Gamyyz * Ayz + Gamzyz * Azz) - chiz * Ayz / chin1;
      azzz = azzz - (Gamxzz * Axz + Gamyzz * Ayz + Gamzzz * Azz + Gamxzz * Axz + Gamyzz * Ayz + Gamzzz * Azz) - chiz * Azz / chin1;
      const T mx = gupxx * axxx + gupyy * axyy + gupzz * axzz + gupxy * axyx + gupxz * axzx + gupyz * axzy +
                   gupxy * axxy + gupxz * axxz + gupyz * axyz;
      const T my = gupxx * axyx + gupyy * ayyy + gupzz * ayzz + gupxy * ayyx + gupxz * ayzx + gupyz * ayzy +
                   gupxy * axyy + gupxz * axyz + gupyz * ayyz;
      const T mz = gupxx * axzx + gupyy * ayzy + gupzz * azzz + gupxy * ayzx + gupxz * azzx + gupyz * azzy +
                   gupxy * axzy + gupxz * axzz + gupyz * ayzz;
      // :1132-1134
      T Kx, Ky, Kz;
      grad<T, F_TRK>(q, C, g.ord, Kx, Ky, Kz);
      o[1 * aux.fs] = mx - F2o3 * Kx - EIGHT * PI * Sx;
      o[2 * aux.fs] = my - F2o3 * Ky - EIGHT * PI * Sy;
      o[3 * aux.fs] = mz - F2o3 * Kz - EIGHT * PI * Sz;
    }
  }
  epi.finish();
  return status;
}

}  // namespace amss
