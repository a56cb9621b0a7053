// interp.cu -- values of fields at arbitrary points of a level
// (Parallel::PatList_Interp_Points, Parallel.C:5614-5667, with
// Patch::Interp_Points, MPatch.C:339-500, and global_interp,
// fmisc.f90:712-794): the host finds the block and the 6^3 stencil of each
// point; one thread per (point, field) gathers the cube (decide3d,
// fmisc.f90:798-874: cells at index <= 0 mirrored times the field's parity)
// and runs Neville's scheme along z, then y, then x (polin3 / polint,
// fmisc.f90:1121-1260) in the Fortran's operation order.  Products go through
// __dmul_rn so that no multiply is fused into the following add.
#include <cuda_runtime.h>

#include "interp.cuh"
#include "amss_common.cuh"

namespace amss {

constexpr int kOrdn = 6;   // 2 * ghost_width

// polint with xa = 0, 1, ..., 5 (fmisc.f90:1121-1179)
__device__ double neville6(const double* ya, double x) {
  double c[kOrdn], d[kOrdn], ho[kOrdn];
  int ns = 1;
  double dif = fabs(x - 0.0);
#pragma unroll
  for (int m = 0; m < kOrdn; ++m) {
    c[m] = ya[m];
    d[m] = ya[m];
    ho[m] = (double)m - x;
    const double dift = fabs(x - (double)m);
    if (dift < dif) {
      ns = m + 1;
      dif = dift;
    }
  }
  double y = ya[ns - 1];
  ns -= 1;
#pragma unroll
  for (int m = 1; m < kOrdn; ++m) {
    double den[kOrdn];
#pragma unroll
    for (int i = 0; i < kOrdn - m; ++i) den[i] = (c[i + 1] - d[i]) / (ho[i] - ho[i + m]);
#pragma unroll
    for (int i = 0; i < kOrdn - m; ++i) d[i] = __dmul_rn(ho[i + m], den[i]);
#pragma unroll
    for (int i = 0; i < kOrdn - m; ++i) c[i] = __dmul_rn(ho[i], den[i]);
    double dy;
    if (2 * ns < kOrdn - m) {
      dy = c[ns];
    } else {
      dy = d[ns - 1];
      ns -= 1;
    }
    y = y + dy;
  }
  return y;
}

// global_interp's cube and polin3 for one field: cxB the first stencil index
// per axis (Fortran numbering; <= 0 mirrored times soa), cx the offsets.
template <typename S>
__device__ double interp_cube(const S* __restrict__ f, const int ex[3], const int cxB[3], const double cx[3],
                              const double soa[3]) {
  const long long sy = ex[0], sz = (long long)ex[0] * ex[1];
  double ym[kOrdn];
  for (int a = 0; a < kOrdn; ++a) {
    const int i = cxB[0] + a;
    const long long oi = (i > 0 ? i : 1 - i) - 1;
    double yat[kOrdn];
    for (int b = 0; b < kOrdn; ++b) {
      const int j = cxB[1] + b;
      const long long oj = (j > 0 ? j : 1 - j) - 1;
      double yq[kOrdn];
#pragma unroll
      for (int c = 0; c < kOrdn; ++c) {
        const int k = cxB[2] + c;
        const long long ok = (k > 0 ? k : 1 - k) - 1;
        double v = (double)f[oi + oj * sy + ok * sz];
        if (i <= 0) v = v * soa[0];
        if (j <= 0) v = v * soa[1];
        if (k <= 0) v = v * soa[2];
        yq[c] = v;
      }
      yat[b] = neville6(yq, cx[2]);
    }
    ym[a] = neville6(yat, cx[1]);
  }
  return neville6(ym, cx[0]);
}

__global__ void __launch_bounds__(64) k_interp_points(const InterpItem* __restrict__ items, int n,
                                                      double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const InterpItem it = items[t];
  out[t] = interp_cube(it.f, it.ex, it.cxB, it.cx, it.soa);
}

// Puncture tracking on the finest level, one RK4 substep (bssn_class.C:3360-3390
// for substep 0, :3730-3760 and :3804-3812 for substeps 1-3, :3890-3898 at the
// end): the right-hand side of each coordinate is minus the shift of the
// substep's input state at the current estimate (compute_Porg_rhs,
// bssn_class.C:6879-6932), advanced by rungekutta4_scalar
// (rungekutta4_rout.f90:6-47).  One CTA per coordinate v of puncture p:
// every thread repeats the (cheap) search, 36 threads run the z passes of
// polin3, 6 the y passes, one the x pass and the update.  Substep k reads the
// estimate of substep k-1 from one buffer and writes the other, so no CTA
// overwrites a coordinate another CTA still reads.
constexpr int kTrackThreads = 64;

__global__ void __launch_bounds__(kTrackThreads) k_track(const TrackPatch* __restrict__ patches, int npatch,
                                                         const TrackBlock* __restrict__ blocks,
                                                         const int* __restrict__ lvl, TrackState* S, int sub,
                                                         double dt, int symmetry) {
  const int p = blockIdx.x / 3, v = blockIdx.x % 3, t = threadIdx.x;
  // estimate in: Porg0 (substep 0), else the previous substep's
  const double* src = sub == 0 ? S->p0 : (sub == 2 ? S->pb : S->pa);
  double pos[3];
  for (int d = 0; d < 3; ++d) pos[d] = src[3 * p + d];
  int blk = -1;
  const bool finite = isfinite(pos[0]) && isfinite(pos[1]) && isfinite(pos[2]);
  for (int q = 0; q < npatch && blk < 0 && finite; ++q) {
    const TrackPatch& P = patches[q];
    bool in = true;
    for (int d = 0; d < 3; ++d)
      if (pos[d] < P.lo[d] || pos[d] > P.hi[d]) in = false;
    if (!in) continue;
    for (int b = P.b0; b < P.b1 && blk < 0; ++b) {
      bool inb = true;
      for (int d = 0; d < 3; ++d)
        if (pos[d] - blocks[b].flo[d] < -P.half[d] || pos[d] - blocks[b].fhi[d] > P.half[d]) inb = false;
      if (inb) blk = b;
    }
    if (blk < 0) break;   // in the patch but in none of its blocks
  }
  __shared__ double yat[kOrdn][kOrdn], ym[kOrdn];
  int cxB[3];
  double cx[3], soa[3];
  const double* f = nullptr;
  if (blk >= 0) {
    const TrackBlock& B = blocks[blk];
    for (int d = 0; d < 3; ++d) {
      const double dd = B.dd[d];
      const int cxI = (int)((pos[d] - B.x0[d]) / dd + 0.4) + 1;
      int lo = cxI - 2, hi = lo + 5;
      if (lo < B.cmin[d]) { lo = B.cmin[d]; hi = lo + 5; }
      if (hi > B.ex[d]) { hi = B.ex[d]; lo = hi - 5; }
      cxB[d] = lo;
      // X(j) of the block, as the host builds its coordinates: bbox_lo + (j - 0.5) h
      const int j = lo > 0 ? lo : 1 - lo;
      const double xj = __dadd_rn(B.blo[d], __dmul_rn((double)(j - 1) + 0.5, B.bh[d]));
      cx[d] = lo > 0 ? (pos[d] - xj) / dd : (pos[d] + xj) / dd;
      soa[d] = d == v ? -1.0 : 1.0;   // beta^v is odd along axis v
    }
    const long long off = (long long)(F_BETAX + v) * B.fs;
    if (sub == 0) {
      f = B.tl[lvl[0]] + off;
    } else if (B.f32) {   // the mixed form's stages hold the shift in their FP64 side slots
      f = B.side[sub == 2 ? 1 : 0] + (long long)(kSideBetaX + v) * B.fs;
    } else {
      f = (const double*)B.stage[sub == 2 ? 1 : 0] + off;
    }
    if (t < kOrdn * kOrdn) {   // polin3's z pass for column (a, b)
      const int a = t / kOrdn, b = t % kOrdn;
      const int i = cxB[0] + a, j = cxB[1] + b;
      const long long oi = (i > 0 ? i : 1 - i) - 1, oj = (j > 0 ? j : 1 - j) - 1;
      const long long sy = B.ex[0], sz = (long long)B.ex[0] * B.ex[1];
      double yq[kOrdn];
#pragma unroll
      for (int c = 0; c < kOrdn; ++c) {
        const int k = cxB[2] + c;
        const long long ok = (k > 0 ? k : 1 - k) - 1;
        const long long o = oi + oj * sy + ok * sz;
        double val = f[o];
        if (i <= 0) val = val * soa[0];
        if (j <= 0) val = val * soa[1];
        if (k <= 0) val = val * soa[2];
        yq[c] = val;
      }
      yat[a][b] = neville6(yq, cx[2]);
    }
  }
  __syncthreads();
  if (blk >= 0 && t < kOrdn) ym[t] = neville6(yat[t], cx[1]);
  __syncthreads();
  if (t != 0) return;
  double R = 0.0;
  if (blk < 0)
    atomicOr(&S->err, 1);
  else
    R = -neville6(ym, cx[0]);
  const int i = 3 * p + v;
  const double p0 = S->p0[i];
  double pn;
  if (sub == 0) {
    S->k[i] = R;
    pn = __dadd_rn(p0, __dmul_rn(__dmul_rn(0.5, dt), R));
  } else if (sub == 1) {
    S->k[i] = __dadd_rn(S->k[i], __dmul_rn(2.0, R));
    pn = __dadd_rn(p0, __dmul_rn(__dmul_rn(0.5, dt), R));
  } else if (sub == 2) {
    S->k[i] = __dadd_rn(S->k[i], __dmul_rn(2.0, R));
    pn = __dadd_rn(p0, __dmul_rn(dt, R));
  } else {
    pn = __dadd_rn(p0, __dmul_rn(__dmul_rn(1.0 / 6.0, dt), __dadd_rn(R, S->k[i])));
  }
  if ((symmetry > 0 && v == 2) || (symmetry == 2 && v < 2)) pn = fabs(pn);
  // estimate out: substeps 0 and 2 write pa, substep 1 pb, substep 3 Porg0
  if (sub == 3)
    S->p0[i] = pn;
  else
    (sub == 1 ? S->pb : S->pa)[i] = pn;
}

cudaError_t launch_track(const TrackPatch* patches, int npatch, const TrackBlock* blocks, const int* lvl,
                         TrackState* S, int n, int sub, double dt, int symmetry, cudaStream_t s) {
  k_track<<<3 * n, kTrackThreads, 0, s>>>(patches, npatch, blocks, lvl, S, sub, dt, symmetry);
  return cudaGetLastError();
}

cudaError_t launch_interp_points(const InterpItem* items, int n, double* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_interp_points<<<(n + 63) / 64, 64, 0, s>>>(items, n, out);
  return cudaGetLastError();
}

}  // namespace amss
