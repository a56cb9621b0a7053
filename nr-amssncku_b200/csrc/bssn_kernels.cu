// bssn_kernels.cu -- BSSN RHS / fused RK4 substep kernels and the drop-in
// C-ABI entry points that replace the reference's per-block Fortran kernels.
//
// Every entry point here takes the reference's arguments (host pointers,
// Fortran order, pass-by-reference scalars), copies them to HBM, runs the
// sm_100a kernel and copies the results back.  None has a CPU fallback: with
// no usable CUDA device they return an error code and say so on stderr.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "bssn_step.cuh"
#include "amss_b200.h"
#include "dropin_ctx.cuh"
#include "dev_util.cuh"
#include "substep_impl.cuh"

namespace amss {

// instantiated in rhs_dropin*.cu
extern template cudaError_t launch_rhs_dropin<false>(int, cudaStream_t, BlockView, Coefs<double>, const double*,
                                                     double*, RhsAux, unsigned*);
extern template cudaError_t launch_rhs_dropin<true>(int, cudaStream_t, BlockView, Coefs<double>, const double*,
                                                    double*, RhsAux, unsigned*);
extern template cudaError_t launch_rhs_dropin_z4c<false>(int, cudaStream_t, BlockView, Coefs<double>, const double*,
                                                         double*, const double*, unsigned*);
extern template cudaError_t launch_rhs_dropin_z4c<true>(int, cudaStream_t, BlockView, Coefs<double>, const double*,
                                                        double*, const double*, unsigned*);

// -----------------------------------------------------------------------------
// Kernels
// -----------------------------------------------------------------------------

// ---- pointwise helper kernels of the drop-in entries -------------------------

__global__ void k_rk4(long long n, double dT, const double* __restrict__ f0, double* f1, double* f_rhs, int RK4) {
  const double F1o6 = 1.0 / 6.0, HLF = 0.5, TWO = 2.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    // explicitly rounded operations (no FMA contraction): the same IEEE
    // operations, in the same order, as the Fortran
    if (RK4 == 0) {
      f1[p] = __dadd_rn(f0[p], __dmul_rn(__dmul_rn(HLF, dT), f_rhs[p]));
    } else if (RK4 == 1) {
      f_rhs[p] = __dadd_rn(f_rhs[p], __dmul_rn(TWO, f1[p]));
      f1[p] = __dadd_rn(f0[p], __dmul_rn(__dmul_rn(HLF, dT), f1[p]));
    } else if (RK4 == 2) {
      f_rhs[p] = __dadd_rn(f_rhs[p], __dmul_rn(TWO, f1[p]));
      f1[p] = __dadd_rn(f0[p], __dmul_rn(dT, f1[p]));
    } else {
      f1[p] = __dadd_rn(f0[p], __dmul_rn(__dmul_rn(F1o6, dT), __dadd_rn(f1[p], f_rhs[p])));
    }
  }
}

__global__ void k_enforce(long long n, long long fs, double* g /* 6 fields */, double* a /* 6 fields */) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    double gv[6], av[6];
    for (int m = 0; m < 6; ++m) { gv[m] = g[m * fs + p]; av[m] = a[m * fs + p]; }
    enforce_ga_point(gv, av);
    for (int m = 0; m < 6; ++m) { g[m * fs + p] = gv[m]; a[m * fs + p] = av[m]; }
  }
}

__global__ void k_floor(long long n, double* chi, double tiny) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
    if (chi[p] < tiny) chi[p] = tiny;
}

// Sommerfeld rule on the face points of one field (one thread per block point,
// face points only do work).
__global__ void k_sommerfeld_field(BlockView b, double d2x, double d2y, double d2z, double* f_rhs,
                                   const double* __restrict__ f0, double velocity, int anti_mask) {
  const long long n = (long long)b.ex[0] * b.ex[1] * b.ex[2];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    point_ijk(p, b.ex, i, j, k);
    const int fm = b.face_mask;
    const bool on_face = ((fm & 1) && i == b.ex[0] - 1) || ((fm & 2) && j == b.ex[1] - 1) ||
                         ((fm & 4) && k == b.ex[2] - 1) || ((fm & 8) && i == 0) || ((fm & 16) && j == 0) ||
                         ((fm & 32) && k == 0);
    if (!on_face) continue;
    const int id[3] = {i, j, k};
    const double xs[3] = {b.X[i], b.Y[j], b.Z[k]};
    const double d2[3] = {d2x, d2y, d2z};
    const double R = sqrt(xs[0] * xs[0] + xs[1] * xs[1] + xs[2] * xs[2]);
    const long long st[3] = {1, b.ex[0], (long long)b.ex[0] * b.ex[1]};
    double fd[3];
    for (int d = 0; d < 3; ++d) {
      const int lo = ((b.lowsym_mask >> d) & 1) ? -1 : 0, hi = b.ex[d] - 1;
      auto f = [&](int o) -> double {
        int m = id[d] + o;
        double sgn = 1.0;
        if (m < 0) { m = -m - 1; if ((anti_mask >> d) & 1) sgn = -1.0; }
        return sgn * f0[p + (long long)(m - id[d]) * st[d]];
      };
      const double w = velocity * xs[d] / R;
      double r = 0.0;
      if (w > 0) {
        if (id[d] - 2 >= lo) r = d2[d] * (3 * f(0) - 4 * f(-1) + f(-2));
        else if (id[d] - 1 >= lo) r = d2[d] * (-f(-1) + f(1));
        else r = d2[d] * (-f(2) + 4 * f(1) - 3 * f(0));
      } else if (w < 0) {
        if (id[d] + 2 <= hi) r = d2[d] * (-f(2) + 4 * f(1) - 3 * f(0));
        else if (id[d] + 1 <= hi) r = d2[d] * (-f(-1) + f(1));
        else r = d2[d] * (3 * f(0) - 4 * f(-1) + f(-2));
      }
      fd[d] = r;
    }
    f_rhs[p] = -velocity * (fd[0] * xs[0] + fd[1] * xs[1] + fd[2] * xs[2] + f0[p]) / R;
  }
}

__global__ void k_freeze_field(BlockView b, const double* __restrict__ f0, double* f) {
  const long long n = (long long)b.ex[0] * b.ex[1] * b.ex[2];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    point_ijk(p, b.ex, i, j, k);
    const int fm = b.face_mask;
    const bool on_face = ((fm & 1) && i == b.ex[0] - 1) || ((fm & 2) && j == b.ex[1] - 1) ||
                         ((fm & 4) && k == b.ex[2] - 1) || ((fm & 8) && i == 0) || ((fm & 16) && j == 0) ||
                         ((fm & 32) && k == 0);
    if (on_face) f[p] = f0[p];
  }
}

// -----------------------------------------------------------------------------
// Host side
// -----------------------------------------------------------------------------

template <typename T>
Coef<T> make_coef(const double dx[3], double eps) {
  const double ONE = 1.0, TWO = 2.0, F12 = 12.0;
  const double F1o12 = ONE / 12.0, F1o144 = ONE / 144.0, F1o4 = 0.25;
  Coef<T> c;
  for (int d = 0; d < 3; ++d) {
    c.d12[d] = (T)(ONE / F12 / dx[d]);
    c.d2[d] = (T)(ONE / TWO / dx[d]);
    c.Fdd[d] = (T)(F1o12 / (dx[d] * dx[d]));
    c.Sdd[d] = (T)(ONE / (dx[d] * dx[d]));
    c.h[d] = (T)dx[d];
    c.hinv[d] = (T)(ONE / dx[d]);
  }
  c.hpow2 = 1;
  for (int d = 0; d < 3; ++d) {
    int e;
    if (!(dx[d] > 0.0) || std::frexp(dx[d], &e) != 0.5) c.hpow2 = 0;
  }
  c.Fxy = (T)(F1o144 / (dx[0] * dx[1]));
  c.Fxz = (T)(F1o144 / (dx[0] * dx[2]));
  c.Fyz = (T)(F1o144 / (dx[1] * dx[2]));
  c.Sxy = (T)(F1o4 / (dx[0] * dx[1]));
  c.Sxz = (T)(F1o4 / (dx[0] * dx[2]));
  c.Syz = (T)(F1o4 / (dx[1] * dx[2]));
  c.ko = (T)(eps > 0 ? eps / 64.0 : 0.0);
  return c;
}
template Coef<double> make_coef<double>(const double*, double);
template Coef<float> make_coef<float>(const double*, double);

// Face mask and symmetry planes of a block, as sommerfeld_rout.f90:56-121 and
// the derivative routines decide them from the coordinates.
void block_faces(const int ex[3], const double* X, const double* Y, const double* Z, const double bbox[6],
                 int symmetry, int* face_mask, int* lowsym_mask) {
  const double dX = X[1] - X[0], dY = Y[1] - Y[0], dZ = Z[1] - Z[0];
  int fm = 0;
  if (std::fabs(X[ex[0] - 1] - bbox[3]) < dX) fm |= 1;
  if (std::fabs(Y[ex[1] - 1] - bbox[4]) < dY) fm |= 2;
  if (std::fabs(Z[ex[2] - 1] - bbox[5]) < dZ) fm |= 4;
  if (std::fabs(X[0] - bbox[0]) < dX && !(symmetry == 2 && std::fabs(bbox[0]) < dX / 2)) fm |= 8;
  if (std::fabs(Y[0] - bbox[1]) < dY && !(symmetry == 2 && std::fabs(bbox[1]) < dY / 2)) fm |= 16;
  if (std::fabs(Z[0] - bbox[2]) < dZ && !(symmetry > 0 && std::fabs(bbox[2]) < dZ / 2)) fm |= 32;
  int ls = 0;
  if (symmetry > 1 && std::fabs(X[0]) < dX) ls |= 1;
  if (symmetry > 1 && std::fabs(Y[0]) < dY) ls |= 2;
  if (symmetry > 0 && std::fabs(Z[0]) < dZ) ls |= 4;
  *face_mask = fm;
  *lowsym_mask = ls;
}

static thread_local DropinCtx g_ctx;
DropinCtx& dropin_ctx() { return g_ctx; }

static int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  const long long cap = 148LL * 16;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace amss

using namespace amss;

// -----------------------------------------------------------------------------
// C ABI: drop-ins for the reference's per-block Fortran kernels
// -----------------------------------------------------------------------------

extern "C" int compute_rhs_bssn_(
    int* ex, double* T, double* X, double* Y, double* Z, double* chi, double* trK, double* dxx, double* gxy,
    double* gxz, double* dyy, double* gyz, double* dzz, double* Axx, double* Axy, double* Axz, double* Ayy,
    double* Ayz, double* Azz, double* Gamx, double* Gamy, double* Gamz, double* Lap, double* betax, double* betay,
    double* betaz, double* dtSfx, double* dtSfy, double* dtSfz, double* chi_rhs, double* trK_rhs, double* gxx_rhs,
    double* gxy_rhs, double* gxz_rhs, double* gyy_rhs, double* gyz_rhs, double* gzz_rhs, double* Axx_rhs,
    double* Axy_rhs, double* Axz_rhs, double* Ayy_rhs, double* Ayz_rhs, double* Azz_rhs, double* Gamx_rhs,
    double* Gamy_rhs, double* Gamz_rhs, double* Lap_rhs, double* betax_rhs, double* betay_rhs, double* betaz_rhs,
    double* dtSfx_rhs, double* dtSfy_rhs, double* dtSfz_rhs, double* rho, double* Sx, double* Sy, double* Sz,
    double* Sxx, double* Sxy, double* Sxz, double* Syy, double* Syz, double* Szz, double* Gamxxx, double* Gamxxy,
    double* Gamxxz, double* Gamxyy, double* Gamxyz, double* Gamxzz, double* Gamyxx, double* Gamyxy, double* Gamyxz,
    double* Gamyyy, double* Gamyyz, double* Gamyzz, double* Gamzxx, double* Gamzxy, double* Gamzxz, double* Gamzyy,
    double* Gamzyz, double* Gamzzz, double* Rxx, double* Rxy, double* Rxz, double* Ryy, double* Ryz, double* Rzz,
    double* ham_Res, double* movx_Res, double* movy_Res, double* movz_Res, double* Gmx_Res, double* Gmy_Res,
    double* Gmz_Res, int* Symmetry, int* Lev, double* eps, int* co) {
  (void)T;
  (void)Lev;
  if (!ex || ex[0] < 3 || ex[1] < 3 || ex[2] < 3) return amss_fail(AMSS_ERR_ARG, "compute_rhs_bssn_: every extent must be >= 3");
  DropinCtx& c = g_ctx;
  if (c.init() != 0) return AMSS_ERR_NO_DEVICE;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  const long long fs = pad_stride(n);
  // layout: 24 state | 10 matter | 24 rhs | 18 gamma | 6 ricci | 7 cons | X Y Z
  const size_t total = (size_t)fs * (24 + 10 + 24 + 18 + 6 + 7) + ex[0] + ex[1] + ex[2] + 8;
  double* d = c.reserve(total);
  if (!d) return amss_fail(AMSS_ERR_CUDA, "compute_rhs_bssn_: device allocation failed");
  double* du = d;
  double* dm = du + 24 * fs;
  double* dr = dm + 10 * fs;
  double* dg = dr + 24 * fs;
  double* dR = dg + 18 * fs;
  double* dc = dR + 6 * fs;
  double* dX = dc + 7 * fs;
  double* dY = dX + ex[0];
  double* dZ = dY + ex[1];
  double* st_in[24] = {chi, trK, dxx, gxy, gxz, dyy, gyz, dzz, Axx, Axy, Axz, Ayy, Ayz, Azz,
                       Gamx, Gamy, Gamz, Lap, betax, betay, betaz, dtSfx, dtSfy, dtSfz};
  double* mat[10] = {rho, Sx, Sy, Sz, Sxx, Sxy, Sxz, Syy, Syz, Szz};
  double* rh[24] = {chi_rhs, trK_rhs, gxx_rhs, gxy_rhs, gxz_rhs, gyy_rhs, gyz_rhs, gzz_rhs,
                    Axx_rhs, Axy_rhs, Axz_rhs, Ayy_rhs, Ayz_rhs, Azz_rhs, Gamx_rhs, Gamy_rhs, Gamz_rhs,
                    Lap_rhs, betax_rhs, betay_rhs, betaz_rhs, dtSfx_rhs, dtSfy_rhs, dtSfz_rhs};
  double* gm[18] = {Gamxxx, Gamxxy, Gamxxz, Gamxyy, Gamxyz, Gamxzz, Gamyxx, Gamyxy, Gamyxz,
                    Gamyyy, Gamyyz, Gamyzz, Gamzxx, Gamzxy, Gamzxz, Gamzyy, Gamzyz, Gamzzz};
  double* rc[6] = {Rxx, Rxy, Rxz, Ryy, Ryz, Rzz};
  double* cs[7] = {ham_Res, movx_Res, movy_Res, movz_Res, Gmx_Res, Gmy_Res, Gmz_Res};
  const size_t bytes = (size_t)n * sizeof(double);
  cudaStream_t s = c.stream;
  for (int f = 0; f < 24; ++f) AMSS_CK(cudaMemcpyAsync(du + f * fs, st_in[f], bytes, cudaMemcpyHostToDevice, s));
  for (int f = 0; f < 10; ++f) AMSS_CK(cudaMemcpyAsync(dm + f * fs, mat[f], bytes, cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dX, X, ex[0] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dY, Y, ex[1] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dZ, Z, ex[2] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemsetAsync(c.dstatus, 0, sizeof(unsigned), s));

  BlockView b{};
  b.ex[0] = ex[0]; b.ex[1] = ex[1]; b.ex[2] = ex[2];
  b.fs = fs;
  b.X = dX; b.Y = dY; b.Z = dZ;
  b.dx[0] = X[1] - X[0]; b.dx[1] = Y[1] - Y[0]; b.dx[2] = Z[1] - Z[0];
  b.symmetry = *Symmetry;
  {
    const double bb[6] = {X[0], Y[0], Z[0], X[ex[0] - 1], Y[ex[1] - 1], Z[ex[2] - 1]};
    block_faces(ex, X, Y, Z, bb, *Symmetry, &b.face_mask, &b.lowsym_mask);
  }
  Coefs<double> C;
  C.t = make_coef<double>(b.dx, *eps);
  C.d = C.t;
  RhsAux aux{dg, dR, dc, dm, fs, *co};
  const int grid = grid_for(n, 128);
  if (b.lowsym_mask) AMSS_CK(launch_rhs_dropin<true>(grid, s, b, C, du, dr, aux, c.dstatus));
  else AMSS_CK(launch_rhs_dropin<false>(grid, s, b, C, du, dr, aux, c.dstatus));
  unsigned hs = 0;
  AMSS_CK(cudaMemcpyAsync(&hs, c.dstatus, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  if ((hs & ST_NAN) || ((hs & ST_PINF) && (hs & ST_NINF))) return 1;  // bssn_rhs.f90:136, outputs untouched
  for (int f = 0; f < 24; ++f) AMSS_CK(cudaMemcpyAsync(rh[f], dr + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  for (int f = 0; f < 18; ++f) AMSS_CK(cudaMemcpyAsync(gm[f], dg + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  for (int f = 0; f < 6; ++f) AMSS_CK(cudaMemcpyAsync(rc[f], dR + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  if (*co == 0)
    for (int f = 0; f < 7; ++f) AMSS_CK(cudaMemcpyAsync(cs[f], dc + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  return 0;
}

extern "C" int compute_rhs_z4c_(
    int* ex, double* T, double* X, double* Y, double* Z, double* chi, double* trK, double* dxx, double* gxy,
    double* gxz, double* dyy, double* gyz, double* dzz, double* Axx, double* Axy, double* Axz, double* Ayy,
    double* Ayz, double* Azz, double* Gamx, double* Gamy, double* Gamz, double* Lap, double* betax, double* betay,
    double* betaz, double* dtSfx, double* dtSfy, double* dtSfz, double* TZ, double* chi_rhs, double* trK_rhs,
    double* gxx_rhs, double* gxy_rhs, double* gxz_rhs, double* gyy_rhs, double* gyz_rhs, double* gzz_rhs,
    double* Axx_rhs, double* Axy_rhs, double* Axz_rhs, double* Ayy_rhs, double* Ayz_rhs, double* Azz_rhs,
    double* Gamx_rhs, double* Gamy_rhs, double* Gamz_rhs, double* Lap_rhs, double* betax_rhs, double* betay_rhs,
    double* betaz_rhs, double* dtSfx_rhs, double* dtSfy_rhs, double* dtSfz_rhs, double* TZ_rhs, double* rho,
    double* Sx, double* Sy, double* Sz, double* Sxx, double* Sxy, double* Sxz, double* Syy, double* Syz, double* Szz,
    double* Gamxxx, double* Gamxxy, double* Gamxxz, double* Gamxyy, double* Gamxyz, double* Gamxzz, double* Gamyxx,
    double* Gamyxy, double* Gamyxz, double* Gamyyy, double* Gamyyz, double* Gamyzz, double* Gamzxx, double* Gamzxy,
    double* Gamzxz, double* Gamzyy, double* Gamzyz, double* Gamzzz, double* Rxx, double* Rxy, double* Rxz,
    double* Ryy, double* Ryz, double* Rzz, double* Hcon, double* Mxcon, double* Mycon, double* Mzcon,
    double* Gmxcon, double* Gmycon, double* Gmzcon, int* Symmetry, int* Lev, double* eps, int* co) {
  (void)T;
  (void)Lev;
  (void)co;   // Z4c_rhs.f90:147: the constraints are always computed
  if (!ex || ex[0] < 3 || ex[1] < 3 || ex[2] < 3) return amss_fail(AMSS_ERR_ARG, "compute_rhs_z4c_: every extent must be >= 3");
  DropinCtx& c = g_ctx;
  if (c.init() != 0) return AMSS_ERR_NO_DEVICE;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  const long long fs = pad_stride(n);
  // layout: 25 state | 10 matter | 25 rhs | 24 scratch rhs | 18 gamma | 6 ricci | 7 cons | X Y Z
  const size_t total = (size_t)fs * (25 + 10 + 25 + 24 + 18 + 6 + 7) + ex[0] + ex[1] + ex[2] + 8;
  double* d = c.reserve(total);
  if (!d) return amss_fail(AMSS_ERR_CUDA, "compute_rhs_z4c_: device allocation failed");
  double* du = d;
  double* dm = du + 25 * fs;
  double* dr = dm + 10 * fs;
  double* dscr = dr + 25 * fs;
  double* dg = dscr + 24 * fs;
  double* dR = dg + 18 * fs;
  double* dc = dR + 6 * fs;
  double* dX = dc + 7 * fs;
  double* dY = dX + ex[0];
  double* dZ = dY + ex[1];
  double* st_in[25] = {chi, trK, dxx, gxy, gxz, dyy, gyz, dzz, Axx, Axy, Axz, Ayy, Ayz, Azz,
                       Gamx, Gamy, Gamz, Lap, betax, betay, betaz, dtSfx, dtSfy, dtSfz, TZ};
  double* mat[10] = {rho, Sx, Sy, Sz, Sxx, Sxy, Sxz, Syy, Syz, Szz};
  double* rh[25] = {chi_rhs, trK_rhs, gxx_rhs, gxy_rhs, gxz_rhs, gyy_rhs, gyz_rhs, gzz_rhs,
                    Axx_rhs, Axy_rhs, Axz_rhs, Ayy_rhs, Ayz_rhs, Azz_rhs, Gamx_rhs, Gamy_rhs, Gamz_rhs,
                    Lap_rhs, betax_rhs, betay_rhs, betaz_rhs, dtSfx_rhs, dtSfy_rhs, dtSfz_rhs, TZ_rhs};
  double* gm[18] = {Gamxxx, Gamxxy, Gamxxz, Gamxyy, Gamxyz, Gamxzz, Gamyxx, Gamyxy, Gamyxz,
                    Gamyyy, Gamyyz, Gamyzz, Gamzxx, Gamzxy, Gamzxz, Gamzyy, Gamzyz, Gamzzz};
  double* rc[6] = {Rxx, Rxy, Rxz, Ryy, Ryz, Rzz};
  double* cs[7] = {Hcon, Mxcon, Mycon, Mzcon, Gmxcon, Gmycon, Gmzcon};
  const size_t bytes = (size_t)n * sizeof(double);
  cudaStream_t s = c.stream;
  for (int f = 0; f < 25; ++f) AMSS_CK(cudaMemcpyAsync(du + f * fs, st_in[f], bytes, cudaMemcpyHostToDevice, s));
  for (int f = 0; f < 10; ++f) AMSS_CK(cudaMemcpyAsync(dm + f * fs, mat[f], bytes, cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dX, X, ex[0] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dY, Y, ex[1] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dZ, Z, ex[2] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemsetAsync(c.dstatus, 0, sizeof(unsigned), s));

  BlockView b{};
  b.ex[0] = ex[0]; b.ex[1] = ex[1]; b.ex[2] = ex[2];
  b.fs = fs;
  b.X = dX; b.Y = dY; b.Z = dZ;
  b.dx[0] = X[1] - X[0]; b.dx[1] = Y[1] - Y[0]; b.dx[2] = Z[1] - Z[0];
  b.symmetry = *Symmetry;
  {
    const double bb[6] = {X[0], Y[0], Z[0], X[ex[0] - 1], Y[ex[1] - 1], Z[ex[2] - 1]};
    block_faces(ex, X, Y, Z, bb, *Symmetry, &b.face_mask, &b.lowsym_mask);
  }
  Coefs<double> C;
  C.t = make_coef<double>(b.dx, *eps);
  C.d = C.t;
  const int grid = grid_for(n, 128);
  // the 25 right-hand sides (Z4c_rhs.f90:126-1265)
  if (b.lowsym_mask) AMSS_CK(launch_rhs_dropin_z4c<true>(grid, s, b, C, du, dr, dm, c.dstatus));
  else AMSS_CK(launch_rhs_dropin_z4c<false>(grid, s, b, C, du, dr, dm, c.dstatus));
  unsigned hs = 0;
  AMSS_CK(cudaMemcpyAsync(&hs, c.dstatus, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  if ((hs & ST_NAN) || ((hs & ST_PINF) && (hs & ST_NINF))) return 1;  // Z4c_rhs.f90:261, outputs untouched
  // ricci_gamma + constraint_bssn (Z4c_rhs.f90:1266-1290): the BSSN diagnostic pass
  // on the first 24 fields, its right-hand sides discarded
  RhsAux aux{dg, dR, dc, dm, fs, 0};
  if (b.lowsym_mask) AMSS_CK(launch_rhs_dropin<true>(grid, s, b, C, du, dscr, aux, c.dstatus));
  else AMSS_CK(launch_rhs_dropin<false>(grid, s, b, C, du, dscr, aux, c.dstatus));
  for (int f = 0; f < 25; ++f) AMSS_CK(cudaMemcpyAsync(rh[f], dr + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  for (int f = 0; f < 18; ++f) AMSS_CK(cudaMemcpyAsync(gm[f], dg + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  for (int f = 0; f < 6; ++f) AMSS_CK(cudaMemcpyAsync(rc[f], dR + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  for (int f = 0; f < 7; ++f) AMSS_CK(cudaMemcpyAsync(cs[f], dc + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  return 0;
}

extern "C" int rungekutta4_rout_(int* ex, double* dT, double* f0, double* f1, double* f_rhs, int* RK4) {
  if (*RK4 < 0 || *RK4 > 3) {
    std::fprintf(stderr, "rungekutta4_rout: something is wrong in RK4 counting!!\n");
    return amss_fail(AMSS_ERR_ARG, "rungekutta4_rout_: RK4 counter out of range");
  }
  DropinCtx& c = g_ctx;
  if (c.init() != 0) return AMSS_ERR_NO_DEVICE;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  const long long fs = pad_stride(n);
  double* d = c.reserve(3 * fs);
  if (!d) return amss_fail(AMSS_ERR_CUDA, "rungekutta4_rout_: device allocation failed");
  const size_t bytes = (size_t)n * sizeof(double);
  cudaStream_t s = c.stream;
  AMSS_CK(cudaMemcpyAsync(d, f0, bytes, cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(d + fs, f1, bytes, cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(d + 2 * fs, f_rhs, bytes, cudaMemcpyHostToDevice, s));
  k_rk4<<<grid_for(n, 256), 256, 0, s>>>(n, *dT, d, d + fs, d + 2 * fs, *RK4);
  AMSS_CK(cudaGetLastError());
  AMSS_CK(cudaMemcpyAsync(f1, d + fs, bytes, cudaMemcpyDeviceToHost, s));
  if (*RK4 == 1 || *RK4 == 2) AMSS_CK(cudaMemcpyAsync(f_rhs, d + 2 * fs, bytes, cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  return 0;
}

extern "C" void enforce_ga_(int* ex, double* dxx, double* gxy, double* gxz, double* dyy, double* gyz, double* dzz,
                            double* Axx, double* Axy, double* Axz, double* Ayy, double* Ayz, double* Azz) {
  DropinCtx& c = g_ctx;
  if (c.init() != 0) return;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  const long long fs = pad_stride(n);
  double* d = c.reserve(12 * fs);
  if (!d) { amss_fail(AMSS_ERR_CUDA, "enforce_ga_: device allocation failed"); return; }
  double* h[12] = {dxx, gxy, gxz, dyy, gyz, dzz, Axx, Axy, Axz, Ayy, Ayz, Azz};
  const size_t bytes = (size_t)n * sizeof(double);
  cudaStream_t s = c.stream;
  for (int f = 0; f < 12; ++f) AMSS_CKV(cudaMemcpyAsync(d + f * fs, h[f], bytes, cudaMemcpyHostToDevice, s));
  k_enforce<<<grid_for(n, 256), 256, 0, s>>>(n, fs, d, d + 6 * fs);
  AMSS_CKV(cudaGetLastError());
  for (int f = 0; f < 12; ++f) AMSS_CKV(cudaMemcpyAsync(h[f], d + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  AMSS_CKV(cudaStreamSynchronize(s));
}

extern "C" void lowerboundset_(int* ex, double* chi, double* tinny) {
  DropinCtx& c = g_ctx;
  if (c.init() != 0) return;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  double* d = c.reserve(pad_stride(n));
  if (!d) { amss_fail(AMSS_ERR_CUDA, "lowerboundset_: device allocation failed"); return; }
  const size_t bytes = (size_t)n * sizeof(double);
  cudaStream_t s = c.stream;
  AMSS_CKV(cudaMemcpyAsync(d, chi, bytes, cudaMemcpyHostToDevice, s));
  k_floor<<<grid_for(n, 256), 256, 0, s>>>(n, d, *tinny);
  AMSS_CKV(cudaGetLastError());
  AMSS_CKV(cudaMemcpyAsync(chi, d, bytes, cudaMemcpyDeviceToHost, s));
  AMSS_CKV(cudaStreamSynchronize(s));
}

static int face_call(int* ex, double* X, double* Y, double* Z, double xmin, double ymin, double zmin, double xmax,
                     double ymax, double zmax, int symmetry, BlockView& b, double*& dbase, long long& fs) {
  DropinCtx& c = g_ctx;
  if (c.init() != 0) return AMSS_ERR_NO_DEVICE;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  fs = pad_stride(n);
  dbase = c.reserve(2 * fs + ex[0] + ex[1] + ex[2] + 8);
  if (!dbase) return amss_fail(AMSS_ERR_CUDA, "sommerfeld: device allocation failed");
  double* dX = dbase + 2 * fs;
  double* dY = dX + ex[0];
  double* dZ = dY + ex[1];
  cudaStream_t s = c.stream;
  AMSS_CK(cudaMemcpyAsync(dX, X, ex[0] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dY, Y, ex[1] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dZ, Z, ex[2] * sizeof(double), cudaMemcpyHostToDevice, s));
  b = BlockView{};
  b.ex[0] = ex[0]; b.ex[1] = ex[1]; b.ex[2] = ex[2];
  b.fs = fs;
  b.X = dX; b.Y = dY; b.Z = dZ;
  b.dx[0] = X[1] - X[0]; b.dx[1] = Y[1] - Y[0]; b.dx[2] = Z[1] - Z[0];
  b.symmetry = symmetry;
  const double bb[6] = {xmin, ymin, zmin, xmax, ymax, zmax};
  block_faces(ex, X, Y, Z, bb, symmetry, &b.face_mask, &b.lowsym_mask);
  return 0;
}

extern "C" void sommerfeld_routbam_(int* ex, double* X, double* Y, double* Z, double* xmin, double* ymin,
                                    double* zmin, double* xmax, double* ymax, double* zmax, double* f_rhs, double* f0,
                                    double* velocity, double* SoA, int* Symmetry) {
  BlockView b;
  double* d;
  long long fs;
  if (face_call(ex, X, Y, Z, *xmin, *ymin, *zmin, *xmax, *ymax, *zmax, *Symmetry, b, d, fs) != 0) return;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  const size_t bytes = (size_t)n * sizeof(double);
  cudaStream_t s = g_ctx.stream;
  AMSS_CKV(cudaMemcpyAsync(d, f_rhs, bytes, cudaMemcpyHostToDevice, s));
  AMSS_CKV(cudaMemcpyAsync(d + fs, f0, bytes, cudaMemcpyHostToDevice, s));
  const int anti = (SoA[0] < 0 ? 1 : 0) | (SoA[1] < 0 ? 2 : 0) | (SoA[2] < 0 ? 4 : 0);
  const double ONE = 1.0, TWO = 2.0;
  k_sommerfeld_field<<<grid_for(n, 256), 256, 0, s>>>(b, ONE / TWO / b.dx[0], ONE / TWO / b.dx[1],
                                                      ONE / TWO / b.dx[2], d, d + fs, *velocity, anti);
  AMSS_CKV(cudaGetLastError());
  AMSS_CKV(cudaMemcpyAsync(f_rhs, d, bytes, cudaMemcpyDeviceToHost, s));
  AMSS_CKV(cudaStreamSynchronize(s));
}

extern "C" void sommerfeld_rout_(int* ex, double* X, double* Y, double* Z, double* xmin, double* ymin, double* zmin,
                                 double* xmax, double* ymax, double* zmax, double* dT, double* chi0, double* Lap0,
                                 double* f0, double* f, double* SoA, int* Symmetry, int* precor) {
  (void)dT; (void)chi0; (void)Lap0; (void)SoA;
  if (*precor != 1) {
    amss_fail(AMSS_ERR_UNSUPPORTED,
              "sommerfeld_rout_: only precor == 1 (freeze the patch faces) is on the evolution path");
    return;
  }
  BlockView b;
  double* d;
  long long fs;
  if (face_call(ex, X, Y, Z, *xmin, *ymin, *zmin, *xmax, *ymax, *zmax, *Symmetry, b, d, fs) != 0) return;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  const size_t bytes = (size_t)n * sizeof(double);
  cudaStream_t s = g_ctx.stream;
  AMSS_CKV(cudaMemcpyAsync(d, f0, bytes, cudaMemcpyHostToDevice, s));
  AMSS_CKV(cudaMemcpyAsync(d + fs, f, bytes, cudaMemcpyHostToDevice, s));
  k_freeze_field<<<grid_for(n, 256), 256, 0, s>>>(b, d, d + fs);
  AMSS_CKV(cudaGetLastError());
  AMSS_CKV(cudaMemcpyAsync(f, d + fs, bytes, cudaMemcpyDeviceToHost, s));
  AMSS_CKV(cudaStreamSynchronize(s));
}

// Explicit instantiations used by the engine (engine.cu).
namespace amss {
cudaError_t launch_enforce(long long n, long long fs, double* g, double* a, cudaStream_t s) {
  const long long b = (n + 255) / 256;
  const int grid = (int)(b < 148LL * 16 ? (b < 1 ? 1 : b) : 148LL * 16);
  k_enforce<<<grid, 256, 0, s>>>(n, fs, g, a);
  return cudaGetLastError();
}
size_t stepblock_size(bool fp32) { return fp32 ? sizeof(StepBlock<float>) : sizeof(StepBlock<double>); }
}  // namespace amss
