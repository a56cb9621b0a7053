// psi4.cu -- the analysis quantities of the engine: the Newman-Penrose scalar
// Psi4 of a level's current state (bssn_class::Compute_Psi4,
// bssn_class.C:6210-6298, with getnp4, getnp4.f90:12-452: Psi4type 0,
// tetradtype 2, ABV 0), the ADM-mass integrand (admmass_bssn), and the host
// side of their surface integrals on a coordinate sphere
// (surface_integral::surf_Wave / surf_MassPAng, surface_integral.C:197-377,
// 2247-2512, GaussInt).
//
// Two passes over the level's points, FP64 from the FP64 state whatever the
// engine's precision: the RHS point function in its diagnostic form writes
// the physical Christoffel symbols and Ricci tensor (what compute_rhs_bssn
// hands getnp4 in the reference) to a scratch array, then the Psi4 pass forms
// the tetrad, D_k K_ij, the electric and magnetic parts and Psi4 into the
// first two fields of each block's RK4 accumulator (free between steps).
#include <cmath>
#include <vector>

#include <cuda_runtime.h>

#include "substep_common.cuh"

namespace amss {

struct EpiDiscard {   // only the diagnostic outputs are wanted
  template <int F>
  __device__ __forceinline__ void put(double) {}
  __device__ __forceinline__ void finish() {}
};

constexpr int kPsi4Threads = 128;

template <typename T, bool SYMM>
__global__ void __launch_bounds__(kPsi4Threads) k_gamricci(const StepBlock<T>* __restrict__ blocks,
                                                           const int2* __restrict__ tiles, int ntiles, int tile_pts,
                                                           double* __restrict__ scr, long long dfs) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
  for (int e = threadIdx.x; e < tile_pts; e += blockDim.x) {
    const int2 tile = tiles[t];
    const StepBlock<T>& B = blocks[tile.x];
    const long long p = (long long)tile.y + e;
    if (p >= B.npts) continue;
    auto q = make_pt<double, SYMM>(B.tl[B.lvl[0]], B.b, p);
    const PointGates G = point_gates(B.b, q.i, q.j, q.k);
    const Coefs<double> C{B.C.d, B.C.d};
    RhsAux aux{scr + B.doff, scr + 18 * dfs + B.doff, nullptr, nullptr, dfs, 1};
    EpiDiscard epi;
    (void)bssn_rhs_point<double, double, SYMM, true>(q, C, G, aux, epi);
  }
}

template <typename T, bool SYMM>
__global__ void __launch_bounds__(kPsi4Threads) k_psi4(const StepBlock<T>* __restrict__ blocks,
                                                       const int2* __restrict__ tiles, int ntiles, int tile_pts,
                                                       const double* __restrict__ scr, long long dfs) {
  const double ONE = 1.0, TWO = 2.0, F1o3 = 1.0 / 3.0, TINYRR = 1.0e-14;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
  for (int e = threadIdx.x; e < tile_pts; e += blockDim.x) {
    const int2 tile = tiles[t];
    const StepBlock<T>& B = blocks[tile.x];
    const long long p = (long long)tile.y + e;
    if (p >= B.npts) continue;
    const double* u = B.tl[B.lvl[0]];
    const long long fs = B.b.fs;
    auto q = make_pt<double, SYMM>(u, B.b, p);
    const PointGates G = point_gates(B.b, q.i, q.j, q.k);
    const Coefs<double> C{B.C.d, B.C.d};
    // fderivs of A~ij, chi, trK (getnp4.f90:346-353), the RHS's gated 4th-order stencils
    double d[8][3];
    grad<double, F_AXX>(q, C, G.ord, d[0][0], d[0][1], d[0][2]);
    grad<double, F_AXY>(q, C, G.ord, d[1][0], d[1][1], d[1][2]);
    grad<double, F_AXZ>(q, C, G.ord, d[2][0], d[2][1], d[2][2]);
    grad<double, F_AYY>(q, C, G.ord, d[3][0], d[3][1], d[3][2]);
    grad<double, F_AYZ>(q, C, G.ord, d[4][0], d[4][1], d[4][2]);
    grad<double, F_AZZ>(q, C, G.ord, d[5][0], d[5][1], d[5][2]);
    grad<double, F_CHI>(q, C, G.ord, d[6][0], d[6][1], d[6][2]);
    grad<double, F_TRK>(q, C, G.ord, d[7][0], d[7][1], d[7][2]);

    const double x = B.b.X[q.i], y = B.b.Y[q.j], z = B.b.Z[q.k];
    const double gxx = u[F_GXX * fs + p] + ONE, gyy = u[F_GYY * fs + p] + ONE, gzz = u[F_GZZ * fs + p] + ONE;
    const double Gxy = u[F_GXY * fs + p], Gxz = u[F_GXZ * fs + p], Gyz = u[F_GYZ * fs + p];
    const double chipn1 = u[F_CHI * fs + p] + ONE;
    // :118-126
    double gupzz = gxx * gyy * gzz + Gxy * Gyz * Gxz + Gxz * Gxy * Gyz - Gxz * gyy * Gxz - Gxy * Gxy * gzz -
                   gxx * Gyz * Gyz;
    const double gupxx = (gyy * gzz - Gyz * Gyz) / gupzz;
    const double gupxy = -(Gxy * gzz - Gyz * Gxz) / gupzz;
    const double gupxz = (Gxy * Gyz - gyy * Gxz) / gupzz;
    const double gupyy = (gxx * gzz - Gxz * Gxz) / gupzz;
    const double gupyz = -(gxx * Gyz - Gxy * Gxz) / gupzz;
    gupzz = (gxx * gyy - Gxy * Gxy) / gupzz;
    // :280-303 tetrad seeds: radial v (index raised), azimuthal u, polar w
    double vx, vy, vz, ux, uy, uz, wx, wy, wz;
    if (fabs(x) < TINYRR && fabs(y) < TINYRR && fabs(z) < TINYRR) {
      vx = TINYRR; vy = TINYRR; vz = TINYRR;
    } else {
      vx = x; vy = y; vz = z;
    }
    if (fabs(x) < TINYRR && fabs(y) < TINYRR) {
      ux = -TINYRR; uy = TINYRR; uz = 0.0;
      wx = TINYRR * z; wy = TINYRR * z; wz = -2 * TINYRR * TINYRR;
    } else {
      ux = -y; uy = x; uz = 0.0;
      wx = x * z; wy = y * z; wz = -(x * x + y * y);
    }
    {
      const double fx = vx, fy = vy, fz = vz;
      vx = gupxx * fx + gupxy * fy + gupxz * fz;
      vy = gupxy * fx + gupyy * fy + gupyz * fz;
      vz = gupxz * fx + gupyz * fy + gupzz * fz;
    }
    const double f = 1.0 / chipn1;
    // :314-344 Gram-Schmidt in the physical metric
    double fx = gxx * vx * vx + gyy * vy * vy + gzz * vz * vz + (Gxy * vx * vy + Gxz * vx * vz + Gyz * vy * vz) * TWO;
    fx = sqrt(fx * f);
    vx = vx / fx; vy = vy / fx; vz = vz / fx;
    fx = gxx * vx * ux + Gxy * vx * uy + Gxz * vx * uz + Gxy * vy * ux + gyy * vy * uy + Gyz * vy * uz +
         Gxz * vz * ux + Gyz * vz * uy + gzz * vz * uz;
    fx = fx * f;
    ux = ux - fx * vx; uy = uy - fx * vy; uz = uz - fx * vz;
    fx = gxx * ux * ux + gyy * uy * uy + gzz * uz * uz + (Gxy * ux * uy + Gxz * ux * uz + Gyz * uy * uz) * TWO;
    fx = sqrt(fx * f);
    ux = ux / fx; uy = uy / fx; uz = uz / fx;
    fx = gxx * vx * wx + Gxy * vx * wy + Gxz * vx * wz + Gxy * vy * wx + gyy * vy * wy + Gyz * vy * wz +
         Gxz * vz * wx + Gyz * vz * wy + gzz * vz * wz;
    fx = fx * f;
    wx = wx - fx * vx; wy = wy - fx * vy; wz = wz - fx * vz;
    fx = gxx * ux * wx + Gxy * ux * wy + Gxz * ux * wz + Gxy * uy * wx + gyy * uy * wy + Gyz * uy * wz +
         Gxz * uz * wx + Gyz * uz * wy + gzz * uz * wz;
    fx = fx * f;
    wx = wx - fx * ux; wy = wy - fx * uy; wz = wz - fx * uz;
    fx = gxx * wx * wx + gyy * wy * wy + gzz * wz * wz + (Gxy * wx * wy + Gxz * wx * wz + Gyz * wy * wz) * TWO;
    fx = sqrt(fx * f);
    wx = wx / fx; wy = wy / fx; wz = wz / fx;

    const double axx = u[F_AXX * fs + p], axy = u[F_AXY * fs + p], axz = u[F_AXZ * fs + p];
    const double ayy = u[F_AYY * fs + p], ayz = u[F_AYZ * fs + p], azz = u[F_AZZ * fs + p];
    const double K = u[F_TRK * fs + p];
    const double chix = d[6][0], chiy = d[6][1], chiz = d[6][2];
    const double tx = d[7][0], ty = d[7][1], tz = d[7][2];
    const double* g = scr + B.doff + p;
    const double Gxxx = g[0], Gxxy = g[dfs], Gxxz = g[2 * dfs], Gxyy = g[3 * dfs], Gxyz = g[4 * dfs], Gxzz = g[5 * dfs];
    const double Gyxx = g[6 * dfs], Gyxy = g[7 * dfs], Gyxz = g[8 * dfs], Gyyy = g[9 * dfs], Gyyz = g[10 * dfs];
    const double Gyzz = g[11 * dfs], Gzxx = g[12 * dfs], Gzxy = g[13 * dfs], Gzxz = g[14 * dfs], Gzyy = g[15 * dfs];
    const double Gzyz = g[16 * dfs], Gzzz = g[17 * dfs];
    const double* r = g + 18 * dfs;
    // :355-390 D_k K_ij up to chi^-1 (D_x K_xx, D_y K_yy, D_z K_zz are not needed by B_ij)
    const double Axxy = d[0][1] - (Gxxy * axx + Gyxy * axy + Gzxy * axz) * TWO - chiy / chipn1 * axx + F1o3 * gxx * ty;
    const double Axxz = d[0][2] - (Gxxz * axx + Gyxz * axy + Gzxz * axz) * TWO - chiz / chipn1 * axx + F1o3 * gxx * tz;
    const double Ayyx = d[3][0] - (Gxxy * axy + Gyxy * ayy + Gzxy * ayz) * TWO - chix / chipn1 * ayy + F1o3 * gyy * tx;
    const double Ayyz = d[3][2] - (Gxyz * axy + Gyyz * ayy + Gzyz * ayz) * TWO - chiz / chipn1 * ayy + F1o3 * gyy * tz;
    const double Azzx = d[5][0] - (Gxxz * axz + Gyxz * ayz + Gzxz * azz) * TWO - chix / chipn1 * azz + F1o3 * gzz * tx;
    const double Azzy = d[5][1] - (Gxyz * axz + Gyyz * ayz + Gzyz * azz) * TWO - chiy / chipn1 * azz + F1o3 * gzz * ty;
    const double Axyx = d[1][0] - (Gxxy * axx + Gyxy * axy + Gzxy * axz + Gxxx * axy + Gyxx * ayy + Gzxx * ayz) -
                        chix / chipn1 * axy + F1o3 * Gxy * tx;
    const double Axyy = d[1][1] - (Gxyy * axx + Gyyy * axy + Gzyy * axz + Gxxy * axy + Gyxy * ayy + Gzxy * ayz) -
                        chiy / chipn1 * axy + F1o3 * Gxy * ty;
    const double Axyz = d[1][2] - (Gxyz * axx + Gyyz * axy + Gzyz * axz + Gxxz * axy + Gyxz * ayy + Gzxz * ayz) -
                        chiz / chipn1 * axy + F1o3 * Gxy * tz;
    const double Axzx = d[2][0] - (Gxxz * axx + Gyxz * axy + Gzxz * axz + Gxxx * axz + Gyxx * ayz + Gzxx * azz) -
                        chix / chipn1 * axz + F1o3 * Gxz * tx;
    const double Axzy = d[2][1] - (Gxyz * axx + Gyyz * axy + Gzyz * axz + Gxxy * axz + Gyxy * ayz + Gzxy * azz) -
                        chiy / chipn1 * axz + F1o3 * Gxz * ty;
    const double Axzz = d[2][2] - (Gxzz * axx + Gyzz * axy + Gzzz * axz + Gxxz * axz + Gyxz * ayz + Gzxz * azz) -
                        chiz / chipn1 * axz + F1o3 * Gxz * tz;
    const double Ayzx = d[4][0] - (Gxxz * axy + Gyxz * ayy + Gzxz * ayz + Gxxy * axz + Gyxy * ayz + Gzxy * azz) -
                        chix / chipn1 * ayz + F1o3 * Gyz * tx;
    const double Ayzy = d[4][1] - (Gxyz * axy + Gyyz * ayy + Gzyz * ayz + Gxyy * axz + Gyyy * ayz + Gzyy * azz) -
                        chiy / chipn1 * ayz + F1o3 * Gyz * ty;
    const double Ayzz = d[4][2] - (Gxzz * axy + Gyzz * ayy + Gzzz * ayz + Gxyz * axz + Gyyz * ayz + Gzyz * azz) -
                        chiz / chipn1 * ayz + F1o3 * Gyz * tz;
    // :392-397 magnetic part, symmetrised
    const double Bxx = (vy * (Axxy - Axyx) + vz * (Axxz - Axzx)) * f;
    const double Byy = (vx * (Ayyx - Axyy) + vz * (Ayyz - Ayzy)) * f;
    const double Bzz = (vx * (Azzx - Axzz) + vy * (Azzy - Ayzz)) * f;
    const double Bxy = (vx * (Axyx - (Axxy + Axyx) / TWO) + vy * (Axyy - Ayyx) / TWO + vz * (Axyz - (Axzy + Ayzx) / TWO)) * f;
    const double Bxz = (vx * (Axzx - (Axxz + Axzx) / TWO) + vy * (Axzy - (Axyz + Ayzx) / TWO) + vz * (Axzz - Azzx) / TWO) * f;
    const double Byz = (vx * (Ayzx - (Axyz + Axzy) / TWO) + vy * (Ayzy - (Ayyz + Ayzy) / TWO) + vz * (Ayzz - Azzy) / TWO) * f;
    // :401-407 K_ij up to chi^-1
    const double Kxx = axx + F1o3 * K * gxx, Kxy = axy + F1o3 * K * Gxy, Kxz = axz + F1o3 * K * Gxz;
    const double Kyy = ayy + F1o3 * K * gyy, Kyz = ayz + F1o3 * K * Gyz, Kzz = azz + F1o3 * K * gzz;
    // :409-435 electric part
    double Exx = gupxx * Kxx * Kxx + gupyy * Kxy * Kxy + gupzz * Kxz * Kxz +
                 TWO * (gupxy * Kxx * Kxy + gupxz * Kxx * Kxz + gupyz * Kxy * Kxz);
    double Eyy = gupxx * Kxy * Kxy + gupyy * Kyy * Kyy + gupzz * Kyz * Kyz +
                 TWO * (gupxy * Kxy * Kyy + gupxz * Kxy * Kyz + gupyz * Kyy * Kyz);
    double Ezz = gupxx * Kxz * Kxz + gupyy * Kyz * Kyz + gupzz * Kzz * Kzz +
                 TWO * (gupxy * Kxz * Kyz + gupxz * Kxz * Kzz + gupyz * Kyz * Kzz);
    double Exy = gupxx * Kxx * Kxy + gupyy * Kxy * Kyy + gupzz * Kxz * Kyz + gupxy * (Kxx * Kyy + Kxy * Kxy) +
                 gupxz * (Kxx * Kyz + Kxz * Kxy) + gupyz * (Kxy * Kyz + Kxz * Kyy);
    double Exz = gupxx * Kxx * Kxz + gupyy * Kxy * Kyz + gupzz * Kxz * Kzz + gupxy * (Kxx * Kyz + Kxy * Kxz) +
                 gupxz * (Kxx * Kzz + Kxz * Kxz) + gupyz * (Kxy * Kzz + Kxz * Kyz);
    double Eyz = gupxx * Kxy * Kxz + gupyy * Kyy * Kyz + gupzz * Kyz * Kzz + gupxy * (Kxy * Kyz + Kyy * Kxz) +
                 gupxz * (Kxy * Kzz + Kyz * Kxz) + gupyz * (Kyy * Kzz + Kyz * Kyz);
    Exx = r[0] - (Exx - Kxx * K) * f - Bxx;
    Exy = r[dfs] - (Exy - Kxy * K) * f - Bxy;
    Exz = r[2 * dfs] - (Exz - Kxz * K) * f - Bxz;
    Eyy = r[3 * dfs] - (Eyy - Kyy * K) * f - Byy;
    Eyz = r[4 * dfs] - (Eyz - Kyz * K) * f - Byz;
    Ezz = r[5 * dfs] - (Ezz - Kzz * K) * f - Bzz;
    // :436-451 m = (u - i w)/sqrt(2)
    const double uuwwxx = ux * ux - wx * wx, uuwwxy = ux * uy - wx * wy, uuwwxz = ux * uz - wx * wz;
    const double uuwwyy = uy * uy - wy * wy, uuwwyz = uy * uz - wy * wz, uuwwzz = uz * uz - wz * wz;
    const double uwxx = ux * wx + wx * ux, uwxy = ux * wy + wx * uy, uwxz = ux * wz + wx * uz;
    const double uwyy = uy * wy + wy * uy, uwyz = uy * wz + wy * uz, uwzz = uz * wz + wz * uz;
    const double rp = Exx * uuwwxx + Eyy * uuwwyy + Ezz * uuwwzz + (Exy * uuwwxy + Exz * uuwwxz + Eyz * uuwwyz) * TWO;
    const double ip = Exx * uwxx + Eyy * uwyy + Ezz * uwzz + (Exy * uwxy + Exz * uwxz + Eyz * uwyz) * TWO;
    B.K[p] = -rp / TWO;
    B.K[fs + p] = -ip / TWO;
  }
}

// admmass_bssn (fadmquantites_bssn.f90:5-65): the integrand of the ADM mass,
// mass^i = (Gam^i / 8 + gup^ij d_j chi / (4 chi^1.25)) / (2 pi) (chi the
// conformal factor, stored less 1), at every point of the level into the
// accumulator's fields 2, 3, 4.  Like the reference's temporaries it is not
// synchronised: a block's ghost cells keep its own values.
template <typename T, bool SYMM>
__global__ void __launch_bounds__(kPsi4Threads) k_admmass(const StepBlock<T>* __restrict__ blocks,
                                                          const int2* __restrict__ tiles, int ntiles, int tile_pts) {
  const double ONE = 1.0, F1o8 = 1.0 / 8.0;
  const double F1o2pi = ONE / (2.0 * M_PI);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
  for (int e = threadIdx.x; e < tile_pts; e += blockDim.x) {
    const int2 tile = tiles[t];
    const StepBlock<T>& B = blocks[tile.x];
    const long long p = (long long)tile.y + e;
    if (p >= B.npts) continue;
    const double* u = B.tl[B.lvl[0]];
    const long long fs = B.b.fs;
    auto q = make_pt<double, SYMM>(u, B.b, p);
    const PointGates G = point_gates(B.b, q.i, q.j, q.k);
    const Coefs<double> C{B.C.d, B.C.d};
    double chix, chiy, chiz;
    grad<double, F_CHI>(q, C, G.ord, chix, chiy, chiz);
    const double gxx = u[F_GXX * fs + p] + ONE, gyy = u[F_GYY * fs + p] + ONE, gzz = u[F_GZZ * fs + p] + ONE;
    const double gxy = u[F_GXY * fs + p], gxz = u[F_GXZ * fs + p], gyz = u[F_GYZ * fs + p];
    double gupzz = gxx * gyy * gzz + gxy * gyz * gxz + gxz * gxy * gyz - gxz * gyy * gxz - gxy * gxy * gzz -
                   gxx * gyz * gyz;
    const double gupxx = (gyy * gzz - gyz * gyz) / gupzz;
    const double gupxy = -(gxy * gzz - gyz * gxz) / gupzz;
    const double gupxz = (gxy * gyz - gyy * gxz) / gupzz;
    const double gupyy = (gxx * gzz - gxz * gxz) / gupzz;
    const double gupyz = -(gxx * gyz - gxy * gxz) / gupzz;
    gupzz = (gxx * gyy - gxy * gxy) / gupzz;
    const double f = 1.0 / 4.0 / pow(u[F_CHI * fs + p] + ONE, 1.25);
    B.K[2 * fs + p] = (F1o8 * u[F_GAMX * fs + p] + f * (gupxx * chix + gupxy * chiy + gupxz * chiz)) * F1o2pi;
    B.K[3 * fs + p] = (F1o8 * u[F_GAMY * fs + p] + f * (gupxy * chix + gupyy * chiy + gupyz * chiz)) * F1o2pi;
    B.K[4 * fs + p] = (F1o8 * u[F_GAMZ * fs + p] + f * (gupxz * chix + gupyz * chiy + gupzz * chiz)) * F1o2pi;
  }
}

template <typename T>
cudaError_t launch_admmass(const void* table, const int2* tiles, int ntiles, int tile_pts, bool symm, cudaStream_t s) {
  const StepBlock<T>* bl = (const StepBlock<T>*)table;
  const int g = ntiles < 148 * 8 ? ntiles : 148 * 8;
  if (symm)
    k_admmass<T, true><<<g, kPsi4Threads, 0, s>>>(bl, tiles, ntiles, tile_pts);
  else
    k_admmass<T, false><<<g, kPsi4Threads, 0, s>>>(bl, tiles, ntiles, tile_pts);
  return cudaGetLastError();
}

template cudaError_t launch_admmass<double>(const void*, const int2*, int, int, bool, cudaStream_t);
template cudaError_t launch_admmass<float>(const void*, const int2*, int, int, bool, cudaStream_t);

// Psi4 of every point of a level into its blocks' accumulators (fields 0, 1);
// scratch holds 24 fields of the level's D layout.
template <typename T>
cudaError_t launch_psi4(const void* table, const int2* tiles, int ntiles, int tile_pts, bool symm, double* scratch,
                        long long dfs, cudaStream_t s) {
  const StepBlock<T>* bl = (const StepBlock<T>*)table;
  const int g = ntiles < 148 * 8 ? ntiles : 148 * 8;
  if (symm) {
    k_gamricci<T, true><<<g, kPsi4Threads, 0, s>>>(bl, tiles, ntiles, tile_pts, scratch, dfs);
    k_psi4<T, true><<<g, kPsi4Threads, 0, s>>>(bl, tiles, ntiles, tile_pts, scratch, dfs);
  } else {
    k_gamricci<T, false><<<g, kPsi4Threads, 0, s>>>(bl, tiles, ntiles, tile_pts, scratch, dfs);
    k_psi4<T, false><<<g, kPsi4Threads, 0, s>>>(bl, tiles, ntiles, tile_pts, scratch, dfs);
  }
  return cudaGetLastError();
}

template cudaError_t launch_psi4<double>(const void*, const int2*, int, int, bool, double*, long long, cudaStream_t);
template cudaError_t launch_psi4<float>(const void*, const int2*, int, int, bool, double*, long long, cudaStream_t);

// ---- host: the sphere and its spin-weighted harmonics ------------------------

// n Gauss-Legendre nodes and weights on [-1, 1] (Newton's iteration on P_n,
// started from cos(pi (i + 3/4) / (n + 1/2)), to a step of 1.2e-16), nodes
// descending: the upper hemisphere (cos theta > 0) first, as the reference
// orders them (misc::gaulegf then misc::inversearray).
void gauss_legendre_desc(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), z1, pp;
    do {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 0; j < n; ++j) {   // P_{j+1} from P_j and P_{j-1}
        const double p3 = p2;
        p2 = p1;
        p1 = ((2 * (double)j + 1) * z * p2 - (double)j * p3) / ((double)j + 1);
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);   // P_n' at the iterate
      z1 = z;
      z = z1 - p1 / pp;
    } while (std::fabs(z - z1) > 1.2e-16);
    x[n - 1 - i] = -z;   // descending: +z in the upper half, -z mirrored
    x[i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

static double factorial(int n) {
  double f = 1.0;
  for (int k = 2; k <= n; ++k) f *= k;
  return f;
}

// Wigner d^l_{m s}(theta) for cos(theta) in [-1, 1] by the explicit sum
// over t of (-1)^t cos^{2l+m-s-2t}(theta/2) sin^{2t+s-m}(theta/2) /
// ((l+m-t)! (l-s-t)! t! (t+s-m)!), times sqrt((l+m)!(l-m)!(l+s)!(l-s)!),
// the terms of even t added first, then those of odd t.
double wigner_d(int l, int m, int s, double costheta) {
  const int c1 = std::max(0, m - s), c2 = std::min(l + m, l - s);
  const double sh = std::sqrt((1 - costheta) / 2.0), ch = std::sqrt((1 + costheta) / 2.0);
  auto term = [&](int t) {
    return std::pow(ch, 2 * l + m - s - 2 * t) * std::pow(sh, 2 * t + s - m) /
           (factorial(l + m - t) * factorial(l - s - t) * factorial(t) * factorial(t + s - m));
  };
  const bool even = (c1 % 2) == 0;   // the sign of the first term
  double v = 0.0;
  for (int t = c1; t <= c2; t += 2) v = even ? v + term(t) : v - term(t);
  for (int t = c1 + 1; t <= c2; t += 2) v = even ? v - term(t) : v + term(t);
  return v * std::sqrt(factorial(l + m) * factorial(l - m) * factorial(l + s) * factorial(l - s));
}

}  // namespace amss
