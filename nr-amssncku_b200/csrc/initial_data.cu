// initial_data.cu -- puncture initial data (get_lousto_nbhs,
// initial_puncture.f90:1970-2202) and its vector-Jacobian product with respect
// to the puncture masses and positions.
//
// psi = 1 + sum_i [u_i + m_i / (2 r_i)], u_i the Bowen-York correction of
// Lousto's approximate solution (zero when the momenta and spins are zero, the
// Brill-Lindquist case), and A_ij the Bowen-York extrinsic curvature of every
// puncture.  Stored as offsets: chi - 1 = psi^-4 - 1, Lap - 1 = psi^-2 - 1,
// A~_ij = A_ij / psi^6; the metric offsets, trK, Gam^i, beta^i, dtSf^i are 0.
// One thread per point, every puncture summed in the reference's order.
#include <cmath>
#include <cstdio>
#include <vector>

#include "amss_b200.h"
#include "amss_common.cuh"
#include "dev_util.cuh"
#include "dropin_ctx.cuh"

namespace amss {

constexpr int kMaxPunctures = 16;

struct Puncture {
  double m, x, y, z, px, py, pz, sx, sy, sz;
};

struct Punctures {
  int n;
  double half_dx;   // the radius used where a cell centre sits on a puncture
  Puncture p[kMaxPunctures];
};

// psi and A_ij (not yet divided by psi^6) at (x, y, z).
__device__ __forceinline__ void lousto_point(const Punctures& P, double x, double y, double z, double& psi,
                                             double A[6]) {
  psi = 1.0;
  for (int m = 0; m < 6; ++m) A[m] = 0.0;
  for (int i = 0; i < P.n; ++i) {
    const Puncture& q = P.p[i];
    double nx = x - q.x, ny = y - q.y, nz = z - q.z;
    double rr = sqrt(nx * nx + ny * ny + nz * nz);
    if (rr < 1e-14) rr = P.half_dx;   // initial_puncture.f90:2022
    nx = nx / rr;
    ny = ny / rr;
    nz = nz / rr;
    const double PP = sqrt(q.px * q.px + q.py * q.py + q.pz * q.pz);
    const double SS = sqrt(q.sx * q.sx + q.sy * q.sy + q.sz * q.sz);
    const double mup = PP > 0.0 ? (q.px * nx + q.py * ny + q.pz * nz) / PP : 0.0;
    const double mus = SS > 0.0 ? (q.sx * nx + q.sy * ny + q.sz * nz) / SS : 0.0;
    const double b = 2.0 * rr / q.m;
    const double l = 1.0 / (1.0 + b);
    const double l2 = l * l, l3 = l2 * l, l4 = l3 * l, l5 = l4 * l;
    // Lousto's expansion coefficients (initial_puncture.f90:2042-2047)
    const double u1 = 5.0 / 8.0 * l * (1.0 - 2.0 * l + 2.0 * l2 - l3 + l4 / 5.0);
    const double u2 =
        (15.0 + 117.0 * l - 79.0 * l2 + 43.0 * l3 - 14.0 * l4 + 2.0 * l5 + 84.0 * log(l) / b) / 40.0 / (b * b);
    const double u3 = l + l2 + l3 - 4.0 * l4 + 2.0 * l5;
    const double u4 = -b * b * l5;
    const double u5 = b * (1.0 + 5.0 * b + 10.0 * b * b) * l5 / 80.0;
    const double ps = (q.py * q.sz - q.pz * q.sy) * nx + (q.pz * q.sx - q.px * q.sz) * ny +
                      (q.px * q.sy - q.py * q.sx) * nz;
    const double u = PP * PP / (q.m * q.m) * (u1 + u2 * (3.0 * mup * mup - 1.0)) +
                     2.0 * SS * SS / 5.0 / (q.m * q.m * q.m * q.m) * (u3 + u4 * (3.0 * mus * mus - 1.0)) + u5 * ps;
    psi = psi + u + 0.5 * q.m / rr;
    // Bowen-York A_ij: momentum part + spin part, times 3 / r^2
    const double pn = q.px * nx + q.py * ny + q.pz * nz;
    const double w = 3.0 / (rr * rr);
    A[0] += (0.5 * (2.0 * q.px * nx - (1.0 - nx * nx) * pn) + 2.0 * nx * (q.sy * nz - q.sz * ny) / rr) * w;
    A[3] += (0.5 * (2.0 * q.py * ny - (1.0 - ny * ny) * pn) + 2.0 * ny * (q.sz * nx - q.sx * nz) / rr) * w;
    A[5] += (0.5 * (2.0 * q.pz * nz - (1.0 - nz * nz) * pn) + 2.0 * nz * (q.sx * ny - q.sy * nx) / rr) * w;
    A[1] += (0.5 * (q.px * ny + nx * q.py + nx * ny * pn) +
             (nx * (q.sz * nx - q.sx * nz) + ny * (q.sy * nz - q.sz * ny)) / rr) * w;
    A[2] += (0.5 * (q.px * nz + nx * q.pz + nx * nz * pn) +
             (nx * (q.sx * ny - q.sy * nx) + nz * (q.sy * nz - q.sz * ny)) / rr) * w;
    A[4] += (0.5 * (q.py * nz + ny * q.pz + ny * nz * pn) +
             (ny * (q.sx * ny - q.sy * nx) + nz * (q.sz * nx - q.sx * nz)) / rr) * w;
  }
}

// The 24 state fields (offsets) of every point, field stride fs.
__global__ void __launch_bounds__(128) k_lousto(int ex0, int ex1, int ex2, const double* __restrict__ X,
                                                const double* __restrict__ Y, const double* __restrict__ Z,
                                                Punctures P, double* __restrict__ out, long long fs) {
  const long long n = (long long)ex0 * ex1 * ex2;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % ex0);
    const int j = (int)((p / ex0) % ex1);
    const int k = (int)(p / ((long long)ex0 * ex1));
    double psi, A[6];
    lousto_point(P, X[i], Y[j], Z[k], psi, A);
    const double p2 = psi * psi;
    const double p6 = p2 * p2 * p2;
    for (int f = 0; f < NFIELDS_BSSN; ++f) out[f * fs + p] = 0.0;
    out[F_CHI * fs + p] = 1.0 / (p2 * p2) - 1.0;
    out[F_LAP * fs + p] = 1.0 / p2 - 1.0;
    out[F_AXX * fs + p] = A[0] / p6;
    out[F_AXY * fs + p] = A[1] / p6;
    out[F_AXZ * fs + p] = A[2] / p6;
    out[F_AYY * fs + p] = A[3] / p6;
    out[F_AYZ * fs + p] = A[4] / p6;
    out[F_AZZ * fs + p] = A[5] / p6;
  }
}

constexpr int kVjpThreads = 256;
constexpr int kVjpBlocks = 148 * 2;

// Brill-Lindquist (zero momenta and spins): with psi = 1 + sum m_i / (2 r_i),
//   dL/dm_i   = sum_p g(p) / (2 r_i),
//   dL/dc_i,d = sum_p g(p) m_i (x_d - c_i,d) / (2 r_i^3),
// g = chi_b (-4 psi^-5) + lap_b (-2 psi^-3).  Per-CTA partial sums
// (4 n values per CTA) in `part`, summed on the host in CTA order.
__global__ void __launch_bounds__(kVjpThreads) k_lousto_vjp(int ex0, int ex1, int ex2, const double* __restrict__ X,
                                                          const double* __restrict__ Y,
                                                          const double* __restrict__ Z, Punctures P,
                                                          const double* __restrict__ chi_b,
                                                          const double* __restrict__ lap_b,
                                                          double* __restrict__ part) {
  __shared__ double red[kVjpThreads / 32][4 * kMaxPunctures];
  double acc[4 * kMaxPunctures];
  for (int m = 0; m < 4 * kMaxPunctures; ++m) acc[m] = 0.0;
  const long long n = (long long)ex0 * ex1 * ex2;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % ex0);
    const int j = (int)((p / ex0) % ex1);
    const int k = (int)(p / ((long long)ex0 * ex1));
    const double x = X[i], y = Y[j], z = Z[k];
    double psi, A[6];
    lousto_point(P, x, y, z, psi, A);
    const double p2 = psi * psi, p3 = p2 * psi;
    const double g = chi_b[p] * (-4.0 / (p3 * p2)) + lap_b[p] * (-2.0 / p3);
#pragma unroll
    for (int q = 0; q < kMaxPunctures; ++q) {
      if (q >= P.n) break;
      const Puncture& c = P.p[q];
      const double dx = x - c.x, dy = y - c.y, dz = z - c.z;
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      if (r < 1e-14) {   // the guarded radius does not depend on the position
        acc[4 * q] += g * 0.5 / P.half_dx;
        continue;
      }
      const double h = g * 0.5 / r;
      const double hp = h * c.m / (r * r);
      acc[4 * q] += h;
      acc[4 * q + 1] += hp * dx;
      acc[4 * q + 2] += hp * dy;
      acc[4 * q + 3] += hp * dz;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < 4 * kMaxPunctures; ++m) {
    if (m >= 4 * P.n) break;
    double v = acc[m];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][m] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4 * P.n) {
    double v = 0.0;
    for (int w = 0; w < kVjpThreads / 32; ++w) v += red[w][threadIdx.x];
    part[(long long)blockIdx.x * 4 * P.n + threadIdx.x] = v;
  }
}

static int grid_of(long long n) {
  const long long b = (n + 127) / 128;
  return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

static int punctures(const char* who, int n, const double* X, const double* Mass, const double* Porg,
                     const double* Pmom, const double* Spin, Punctures& P) {
  if (n < 0 || n > kMaxPunctures) {
    char m[160];
    std::snprintf(m, sizeof m, "%s: %d punctures (at most %d)", who, n, kMaxPunctures);
    return amss_fail(AMSS_ERR_ARG, m);
  }
  P.n = n;
  P.half_dx = (X[1] - X[0]) / 2.0;
  for (int i = 0; i < n; ++i) {
    Puncture& q = P.p[i];
    q.m = Mass[i];
    q.x = Porg[3 * i];
    q.y = Porg[3 * i + 1];
    q.z = Porg[3 * i + 2];
    q.px = Pmom ? Pmom[3 * i] : 0.0;
    q.py = Pmom ? Pmom[3 * i + 1] : 0.0;
    q.pz = Pmom ? Pmom[3 * i + 2] : 0.0;
    q.sx = Spin ? Spin[3 * i] : 0.0;
    q.sy = Spin ? Spin[3 * i + 1] : 0.0;
    q.sz = Spin ? Spin[3 * i + 2] : 0.0;
  }
  return 0;
}

}  // namespace amss

using namespace amss;

extern "C" int get_lousto_nbhs_(int* ex, double* X, double* Y, double* Z, double* chi, double* trK, double* gxx,
                                double* gxy, double* gxz, double* gyy, double* gyz, double* gzz, double* Axx,
                                double* Axy, double* Axz, double* Ayy, double* Ayz, double* Azz, double* Gmx,
                                double* Gmy, double* Gmz, double* Lap, double* Sfx, double* Sfy, double* Sfz,
                                double* dtSfx, double* dtSfy, double* dtSfz, double* Mass, double* Porg,
                                double* Pmom, double* Spin, int* N) {
  if (!ex || ex[0] < 2 || ex[1] < 1 || ex[2] < 1 || !N)
    return amss_fail(AMSS_ERR_ARG, "get_lousto_nbhs_: needs ex[0] >= 2 (the cell size is X(2) - X(1))");
  Punctures P{};
  if (int rc = punctures("get_lousto_nbhs_", *N, X, Mass, Porg, Pmom, Spin, P)) return rc;
  DropinCtx& c = dropin_ctx();
  if (c.init() != 0) return AMSS_ERR_NO_DEVICE;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  const long long fs = pad_stride(n);
  const long long nc = ex[0] + ex[1] + ex[2];
  double* d = c.reserve((size_t)NFIELDS_BSSN * fs + nc);
  if (!d) return amss_fail(AMSS_ERR_CUDA, "get_lousto_nbhs_: device allocation failed");
  double* dX = d + (size_t)NFIELDS_BSSN * fs;
  cudaStream_t s = c.stream;
  AMSS_CK(cudaMemcpyAsync(dX, X, ex[0] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dX + ex[0], Y, ex[1] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dX + ex[0] + ex[1], Z, ex[2] * sizeof(double), cudaMemcpyHostToDevice, s));
  k_lousto<<<grid_of(n), 128, 0, s>>>(ex[0], ex[1], ex[2], dX, dX + ex[0], dX + ex[0] + ex[1], P, d, fs);
  AMSS_CK(cudaGetLastError());
  double* h[NFIELDS_BSSN] = {chi, trK, gxx, gxy, gxz, gyy, gyz, gzz, Axx, Axy, Axz, Ayy,
                             Ayz, Azz, Gmx, Gmy, Gmz, Lap, Sfx, Sfy, Sfz, dtSfx, dtSfy, dtSfz};
  for (int f = 0; f < NFIELDS_BSSN; ++f)
    AMSS_CK(cudaMemcpyAsync(h[f], d + f * fs, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  return 0;
}

extern "C" int amss_lousto_vjp(const int* ex, const double* X, const double* Y, const double* Z, int N,
                               const double* Mass, const double* Porg, const double* chi_b, const double* lap_b,
                               double* dMass, double* dPorg) {
  if (!ex || ex[0] < 2 || ex[1] < 1 || ex[2] < 1 || !chi_b || !lap_b || !dMass || !dPorg)
    return amss_fail(AMSS_ERR_ARG, "amss_lousto_vjp: bad arguments");
  Punctures P{};
  if (int rc = punctures("amss_lousto_vjp", N, X, Mass, Porg, nullptr, nullptr, P)) return rc;
  DropinCtx& c = dropin_ctx();
  if (c.init() != 0) return AMSS_ERR_NO_DEVICE;
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  const long long fs = pad_stride(n);
  const long long nc = ex[0] + ex[1] + ex[2];
  const long long np = (long long)kVjpBlocks * 4 * kMaxPunctures;
  double* d = c.reserve(2 * fs + nc + np);
  if (!d) return amss_fail(AMSS_ERR_CUDA, "amss_lousto_vjp: device allocation failed");
  double* dX = d + 2 * fs;
  double* part = dX + nc;
  cudaStream_t s = c.stream;
  AMSS_CK(cudaMemcpyAsync(d, chi_b, n * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(d + fs, lap_b, n * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dX, X, ex[0] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dX + ex[0], Y, ex[1] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dX + ex[0] + ex[1], Z, ex[2] * sizeof(double), cudaMemcpyHostToDevice, s));
  k_lousto_vjp<<<kVjpBlocks, kVjpThreads, 0, s>>>(ex[0], ex[1], ex[2], dX, dX + ex[0], dX + ex[0] + ex[1], P, d,
                                                  d + fs, part);
  AMSS_CK(cudaGetLastError());
  std::vector<double> h((size_t)kVjpBlocks * 4 * N);
  if (N > 0) AMSS_CK(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  for (int q = 0; q < N; ++q) {
    double a[4] = {0, 0, 0, 0};
    for (int b = 0; b < kVjpBlocks; ++b)
      for (int m = 0; m < 4; ++m) a[m] += h[(size_t)b * 4 * N + 4 * q + m];
    dMass[q] = a[0];
    for (int d3 = 0; d3 < 3; ++d3) dPorg[3 * q + d3] = a[1 + d3];
  }
  return 0;
}
