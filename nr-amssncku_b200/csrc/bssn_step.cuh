// bssn_step.cuh -- epilogues and point operations of the fused RK4 substep.
//
// The reference runs, per block and RK4 substep (bssn_class.C:3043-3158 and
// :3401-3525): enforce_ga on the stage input, compute_rhs_bssn,
// sommerfeld_routbam (level 0) on each RHS, rungekutta4_rout, sommerfeld_rout
// with precor=1 (levels > 0, freezes the outer faces at U0) and
// lowerboundset.  Here one kernel launch does all of it per point:
//
//   stage input --stencils--> RHS k --RK4 update--> face rule --> chi floor
//   --> enforce_ga --> stage output
//
// enforce_ga of the stage outputs of substeps 0-2 is applied as they are
// written rather than by a pass before the next substep reads them: it is
// pointwise, so enforce_ga(floor(rk(x))) at a point equals the reference's
// "write, then enforce in place before the next RHS".  The new state written
// by substep 3 is left as the reference leaves it; the engine enforces it in
// place at the start of the next step, after the AMR transfers have run, as
// the reference does.
#pragma once
#include "bssn_rhs.cuh"

namespace amss {

// enforce_algebra.f90:72-133 on one point (double; a recording scalar type for
// the adjoint generator).
template <typename T = double>
__device__ __forceinline__ void enforce_ga_point(T* g, T* a) {
  // g = {dxx, gxy, gxz, dyy, gyz, dzz}, a = {Axx, Axy, Axz, Ayy, Ayz, Azz}
  const double F1o3 = 1.0 / 3.0, ONE = 1.0, TWO = 2.0;
  T gxx = g[0] + ONE, gyy = g[3] + ONE, gzz = g[5] + ONE;
  T gxy = g[1], gxz = g[2], gyz = g[4];
  T d = gxx * gyy * gzz + gxy * gyz * gxz + gxz * gxy * gyz - gxz * gyy * gxz - gxy * gxy * gzz - gxx * gyz * gyz;
  d = ONE / pow(d, F1o3);
  gxx = gxx * d; gxy = gxy * d; gxz = gxz * d; gyy = gyy * d; gyz = gyz * d; gzz = gzz * d;
  g[0] = gxx - ONE; g[1] = gxy; g[2] = gxz; g[3] = gyy - ONE; g[4] = gyz; g[5] = gzz - ONE;
  const T uxx = (gyy * gzz - gyz * gyz);
  const T uxy = -(gxy * gzz - gyz * gxz);
  const T uxz = (gxy * gyz - gyy * gxz);
  const T uyy = (gxx * gzz - gxz * gxz);
  const T uyz = -(gxx * gyz - gxy * gxz);
  const T uzz = (gxx * gyy - gxy * gxy);
  const T trA = uxx * a[0] + uyy * a[3] + uzz * a[5] + TWO * (uxy * a[1] + uxz * a[2] + uyz * a[4]);
  a[0] = a[0] - F1o3 * gxx * trA;
  a[1] = a[1] - F1o3 * gxy * trA;
  a[2] = a[2] - F1o3 * gxz * trA;
  a[3] = a[3] - F1o3 * gyy * trA;
  a[4] = a[4] - F1o3 * gyz * trA;
  a[5] = a[5] - F1o3 * gzz * trA;
}

// Store epilogue: the RHS itself (drop-in compute_rhs_bssn_).
template <typename T>
struct EpiStore {
  double* rhs;
  long long fs, p;
  template <int F>
  __device__ __forceinline__ void put(T v) { rhs[F * fs + p] = (double)v; }
  __device__ __forceinline__ void finish() {}
};

// Substep constants (rungekutta4_rout.f90:94-139 with the products the
// Fortran forms, evaluated once on the host).
struct RKConst {
  double half_dt;   // HLF * dT
  double dt;        // dT
  double sixth_dt;  // F1o6 * dT
  double chitiny;   // lowerboundset threshold (chitiny - 1)
};

// RK4 epilogue: fused update of one field at one point.
template <typename T, typename SO>
struct EpiRK {
  const double* u0;   // state at t_n (FP64)
  double* K;          // RK accumulator (FP64)
  SO* out;            // stage output, or the new state at sub == 3
  double* out_side;   // FP64 side slots (chi, alpha, beta^i) of an FP32 stage output
  long long fs, p;
  int sub;
  bool freeze;        // outer face of a refined patch: output = u0 there
  bool enforce;
  RKConst c;
  double g[6], a[6];

  template <int F>
  __device__ __forceinline__ void put(T kv) {
    const long long o = F * fs + p;
    const double k = (double)kv;
    const double u = u0[o];
    double r;
    if (freeze) {
      // a frozen point's accumulator is never read (it would only feed r)
      r = u;
    } else if (sub == 0) {
      r = u + c.half_dt * k;
      K[o] = k;
    } else if (sub == 1) {
      K[o] = K[o] + 2.0 * k;
      r = u + c.half_dt * k;
    } else if (sub == 2) {
      K[o] = K[o] + 2.0 * k;
      r = u + c.dt * k;
    } else {
      r = u + c.sixth_dt * (k + K[o]);
    }
    if constexpr (F == F_CHI) {
      if (r < c.chitiny) r = c.chitiny;
    }
    if constexpr (F == F_GXX) g[0] = r;
    else if constexpr (F == F_GXY) g[1] = r;
    else if constexpr (F == F_GXZ) g[2] = r;
    else if constexpr (F == F_GYY) g[3] = r;
    else if constexpr (F == F_GYZ) g[4] = r;
    else if constexpr (F == F_GZZ) g[5] = r;
    else if constexpr (F == F_AXX) a[0] = r;
    else if constexpr (F == F_AXY) a[1] = r;
    else if constexpr (F == F_AXZ) a[2] = r;
    else if constexpr (F == F_AYY) a[3] = r;
    else if constexpr (F == F_AYZ) a[4] = r;
    else if constexpr (F == F_AZZ) a[5] = r;
    else if constexpr (sizeof(SO) == 4 && wide_field<F>()) out_side[side_slot(F) * fs + p] = r;
    else out[o] = (SO)r;
  }
  __device__ __forceinline__ void finish() {
    if (enforce) enforce_ga_point(g, a);
    out[F_GXX * fs + p] = (SO)g[0]; out[F_GXY * fs + p] = (SO)g[1]; out[F_GXZ * fs + p] = (SO)g[2];
    out[F_GYY * fs + p] = (SO)g[3]; out[F_GYZ * fs + p] = (SO)g[4]; out[F_GZZ * fs + p] = (SO)g[5];
    out[F_AXX * fs + p] = (SO)a[0]; out[F_AXY * fs + p] = (SO)a[1]; out[F_AXZ * fs + p] = (SO)a[2];
    out[F_AYY * fs + p] = (SO)a[3]; out[F_AYZ * fs + p] = (SO)a[4]; out[F_AZZ * fs + p] = (SO)a[5];
  }
};

// Sommerfeld RHS of one field at an outer-face point
// (sommerfeld_rout.f90:378-440, "new code, 2012dec26"):
//   rhs = -v (x fx + y fy + z fz + f) / r, one-sided 2nd order, upwinded by
//   the sign of v x_d / r.  imin/imax are 0-based; lo = -1 at a symmetry plane.
template <typename T, int F, typename P>
__device__ __forceinline__ T sommerfeld_point(const P& q, const T (&d2)[3], const int (&lo)[3], const int (&hi)[3],
                                             T x, T y, T z, T velocity) {
  const T R = sqrt(x * x + y * y + z * z);
  const T w[3] = {velocity * x / R, velocity * y / R, velocity * z / R};
  const int id[3] = {q.i, q.j, q.k};
  T fd[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    auto f = [&](int o) -> T {
      return q.template vpad<T, F>(d == 0 ? o : 0, d == 1 ? o : 0, d == 2 ? o : 0);
    };
    T r = T(0);
    if (w[d] > T(0)) {
      if (id[d] - 2 >= lo[d]) r = d2[d] * (T(3) * f(0) - T(4) * f(-1) + f(-2));
      else if (id[d] - 1 >= lo[d]) r = d2[d] * (-f(-1) + f(1));
      else r = d2[d] * (-f(2) + T(4) * f(1) - T(3) * f(0));
    } else if (w[d] < T(0)) {
      if (id[d] + 2 <= hi[d]) r = d2[d] * (-f(2) + T(4) * f(1) - T(3) * f(0));
      else if (id[d] + 1 <= hi[d]) r = d2[d] * (-f(-1) + f(1));
      else r = d2[d] * (T(3) * f(0) - T(4) * f(-1) + f(-2));
    }
    fd[d] = r;
  }
  const T f0 = q.template v<T, F>(0, 0, 0);
  return -velocity * (fd[0] * x + fd[1] * y + fd[2] * z + f0) / R;
}

// One block of a level as the fused substep sees it.
template <typename T>
struct StepBlock {
  BlockView b;
  Coefs<T> C;
  T d2s[3];           // 1/2/dx for the Sommerfeld rule
  double* tl[3];      // three time levels of the FP64 state: tl[cur] = U0 (t_n),
                      // tl[(cur+1)%3] receives U_new (it held t_n - 2 dt)
  const int* lvl;     // level state {cur, steps taken} (device, rotated after each step)
  void* stage[2];     // stage buffers A and B (type of the stage storage)
  double* side[2];    // FP64 side slots (chi, alpha, beta^i) of stages A and B (mixed form only)
  double* K;          // RK accumulator (FP64)
  long long doff;     // offset of this block's points in the level's D slots (split form)
  long long npts;
  int lev0;           // 1: Sommerfeld rule on the patch faces; 0: freeze them at u0
  int nf;             // evolved fields: 24 (BSSN) or 25 (Z4c, Theta last)
  int dw;             // stencil-pass tile width (deriv_tile_w of ex[0])
  // regions of region tiles, array indices [rlo, rlo + rn): [0] the final
  // substep's, [1] the block's owned cells (its ghosts are synchronised)
  int rlo[2][3], rn[2][3];
};

// Tile of a pointwise list: tile.x = table index, tile.y = first point.
// With kRegionTile set in tile.x, the points count one of the block's regions
// in x-fastest order instead of its whole array: the final substep's, or with
// kOwnRegion also set its owned cells.
constexpr int kRegionTile = 1 << 30;
constexpr int kOwnRegion = 1 << 29;
constexpr int kTileIndex = kOwnRegion - 1;

}  // namespace amss
