// amr.cuh -- device side of the AMR data movement (ghost sync, restriction,
// prolongation, time interpolation) between blocks resident in HBM.
//
// Every operation is a list of boxes in global level indices; a box names a
// destination block and a source block.  Threads are mapped to box points
// through a tile list (128 points per tile), so one launch serves all boxes
// of a level, whatever their sizes.  Each thread moves all nf fields of one
// point.  Nothing here applies enforce_ga: as in the reference, restricted and
// prolonged values are enforced by the pass at the start of the next step.
#pragma once
#include "amr_types.cuh"

namespace amss {

__device__ __forceinline__ long long amr_idx(const AmrBlock& b, int gi, int gj, int gk) {
  return (long long)(gi - b.org[0]) + (long long)b.ex[0] * ((long long)(gj - b.org[1]) + (long long)b.ex[1] * (gk - b.org[2]));
}
__device__ __forceinline__ bool amr_inside(const AmrBlock& b, int gi, int gj, int gk) {
  return gi >= b.org[0] && gi < b.org[0] + b.ex[0] && gj >= b.org[1] && gj < b.org[1] + b.ex[1] &&
         gk >= b.org[2] && gk < b.org[2] + b.ex[2];
}
__device__ __forceinline__ double* amr_state(const AmrBlock& b) { return b.tl[b.lvl[0]]; }

// Same-level ghost fill: copy the nf fields of each box point from src to dst.
template <typename SS>
__global__ void k_amr_sync(const AmrBlock* __restrict__ blocks, const AmrBox* __restrict__ boxes,
                           const int2* __restrict__ tiles, int ntiles, int which, unsigned* status) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 tile = tiles[t];
    const AmrBox& bx = boxes[tile.x];
    const int p = tile.y + threadIdx.x;
    const int np = bx.n[0] * bx.n[1] * bx.n[2];
    if (p >= np) continue;
    const int gi = bx.lo[0] + p % bx.n[0], gj = bx.lo[1] + (p / bx.n[0]) % bx.n[1], gk = bx.lo[2] + p / (bx.n[0] * bx.n[1]);
    const AmrBlock& D = blocks[bx.dst];
    const AmrBlock& S = blocks[bx.src];
    if (!amr_inside(D, gi, gj, gk) || !amr_inside(S, gi, gj, gk)) { atomicOr(status, ST_BAD_ARG); continue; }
    const long long od = amr_idx(D, gi, gj, gk), os = amr_idx(S, gi, gj, gk);
    if (which == BUF_STATE || which == BUF_TEMP) {
      const double* s = which == BUF_STATE ? amr_state(S) : S.K;
      double* d = which == BUF_STATE ? amr_state(D) : D.K;
      for (int f = 0; f < D.nf; ++f) d[f * D.fs + od] = s[f * S.fs + os];
    } else {
      const int sl = which == BUF_STAGE_A ? 0 : 1;
      const SS* s = (const SS*)S.st[sl];
      SS* d = (SS*)D.st[sl];
      for (int f = 0; f < D.nf; ++f) d[f * D.fs + od] = s[f * S.fs + os];
      if constexpr (sizeof(SS) == 4) {
        for (int f = 0; f < kSideFields; ++f) D.side[sl][f * D.fs + od] = S.side[sl][f * S.fs + os];
      }
    }
  }
}

// prolongrestrict_cell.f90:1937-1942 and :2350
__device__ __constant__ double kProlongW[6] = {7.7e1 / 8.192e3, -6.93e2 / 8.192e3, 3.465e3 / 4.096e3,
                                               1.155e3 / 4.096e3, -4.95e2 / 8.192e3, 6.3e1 / 8.192e3};

// Fine buffer cells of dst (fine) from the parent level's src block:
// prolong3 (prolongrestrict_cell.f90:1915-2164), z then y then x; g odd is
// the right child of k = g >> 1 (coarse k-2..k+3, weights C1..C6), g even
// the left child (coarse k-3..k+2, weights C6..C1).
//
// One thread takes one field of a run of kProlongRun fine cells along x that
// starts at an even index (cells outside the box are skipped).  The cells of a
// run share their y and z weights, so the z-then-y reduction of each coarse x
// column the run reads is formed once (14 columns for 16 cells instead of 6
// per cell) and the x sums of the cells reuse it: the same operations in the same
// order as the cell-by-cell form.  Tiles count (field, run) units, field-major
// within a box, not cells.
__global__ void k_amr_prolong(const AmrBlock* __restrict__ blocks, const AmrBox* __restrict__ boxes,
                              const int2* __restrict__ tiles, int ntiles, int from_temp, unsigned* status) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 tile = tiles[t];
    const AmrBox& bx = boxes[tile.x];
    const int nrx = prolong_runs_x(bx.lo[0], bx.n[0]);
    const int nru = nrx * bx.n[1] * bx.n[2];
    const AmrBlock& D = blocks[bx.dst];
    const int uu = tile.y + threadIdx.x;
    if (uu >= nru * D.nf) continue;
    const int f = uu / nru, u = uu - f * nru;
    const int xs = (bx.lo[0] & ~1) + (u % nrx) * kProlongRun;   // even first fine x of the run
    const int gy = bx.lo[1] + (u / nrx) % bx.n[1], gz = bx.lo[2] + u / (nrx * bx.n[1]);
    const int xlo = bx.lo[0], xhi = bx.lo[0] + bx.n[0];
    const AmrBlock& S = blocks[bx.src];
    const bool ry = (gy & 1) == 0, rz = (gz & 1) == 0;
    const int sy0 = ry ? (gy >> 1) - 3 : (gy >> 1) - 2;
    const int sz0 = rz ? (gz >> 1) - 3 : (gz >> 1) - 2;
    const int cx0 = (xs >> 1) - 3;   // coarse x column of T[0]
    // every source cell of the run, and every destination cell, must exist
    const int first = xs < xlo ? xlo : xs, last = (xs + kProlongRun < xhi ? xs + kProlongRun : xhi) - 1;
    const int c_first = (first & 1) ? (first >> 1) - 2 : (first >> 1) - 3;
    const int c_last = ((last & 1) ? (last >> 1) - 2 : (last >> 1) - 3) + 5;
    if (!amr_inside(D, first, gy, gz) || !amr_inside(D, last, gy, gz) || !amr_inside(S, c_first, sy0, sz0) ||
        !amr_inside(S, c_last, sy0 + 5, sz0 + 5)) {
      atomicOr(status, ST_BAD_ARG);
      continue;
    }
    const double* src = from_temp ? S.K : amr_state(S);
    const long long sy = S.ex[0], sz = (long long)S.ex[0] * S.ex[1];
    double wy[6], wz[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      wy[m] = kProlongW[ry ? 5 - m : m];
      wz[m] = kProlongW[rz ? 5 - m : m];
    }
    double* dst = amr_state(D);
    const long long od0 = amr_idx(D, xs, gy, gz);
    // columns the run reads: T[c] for coarse x = cx0 + c, c in [c_first - cx0, c_last - cx0]
    const int cb = c_first - cx0, ce = c_last - cx0;
    {
      const double* q = src + f * S.fs;
      double T[kProlongRun / 2 + 6];
#pragma unroll
      for (int c = 0; c < kProlongRun / 2 + 6; ++c) {
        T[c] = 0.0;
        if (c < cb || c > ce) continue;
        const long long base = amr_idx(S, cx0 + c, sy0, sz0);
        double t1 = 0.0;
#pragma unroll
        for (int b = 0; b < 6; ++b) {
          const double* r = q + base + b * sy;
          double t2 = __dmul_rn(wz[0], r[0]);
#pragma unroll
          for (int m = 1; m < 6; ++m) t2 = __dadd_rn(t2, __dmul_rn(wz[m], r[m * sz]));
          t1 = b == 0 ? __dmul_rn(wy[0], t2) : __dadd_rn(t1, __dmul_rn(wy[b], t2));
        }
        T[c] = t1;
      }
#pragma unroll
      for (int i = 0; i < kProlongRun; ++i) {
        const int gx = xs + i;
        if (gx < xlo || gx >= xhi) continue;
        // even i: left child, coarse columns i/2 .. i/2 + 5 of T with weights C6..C1;
        // odd i: right child, columns i/2 + 1 .. i/2 + 6 with C1..C6
        const int c0 = (i & 1) ? i / 2 + 1 : i / 2;
        double v = 0.0;
#pragma unroll
        for (int a = 0; a < 6; ++a) {
          const double w = kProlongW[(i & 1) ? a : 5 - a];
          v = a == 0 ? __dmul_rn(w, T[c0]) : __dadd_rn(v, __dmul_rn(w, T[c0 + a]));
        }
        dst[f * D.fs + od0 + i] = v;
      }
    }
  }
}

// Coarse cells of dst (coarse) from fine src: restrict3
// (prolongrestrict_cell.f90:2330-2468): fine 2k-2..2k+3 with weights
// C1 C2 C3 C3 C2 C1, z then y then x.  Writes the current state or the
// time-interpolated temp.  One thread per (field, coarse cell) unit,
// field-major within a box, so consecutive threads take consecutive cells.
__global__ void k_amr_restrict(const AmrBlock* __restrict__ blocks, const AmrBox* __restrict__ boxes,
                               const int2* __restrict__ tiles, int ntiles, int to_temp, unsigned* status) {
  const double C1 = 3.0 / 2.56e2, C2 = -2.5e1 / 2.56e2, C3 = 7.5e1 / 1.28e2;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 tile = tiles[t];
    const AmrBox& bx = boxes[tile.x];
    const AmrBlock& D = blocks[bx.dst];
    const int np = bx.n[0] * bx.n[1] * bx.n[2];
    const int uu = tile.y + threadIdx.x;
    if (uu >= np * D.nf) continue;
    const int f = uu / np, p = uu - f * np;
    const int c[3] = {bx.lo[0] + p % bx.n[0], bx.lo[1] + (p / bx.n[0]) % bx.n[1], bx.lo[2] + p / (bx.n[0] * bx.n[1])};
    const AmrBlock& S = blocks[bx.src];
    const int f0[3] = {2 * c[0] - 2, 2 * c[1] - 2, 2 * c[2] - 2};
    if (!amr_inside(D, c[0], c[1], c[2]) || !amr_inside(S, f0[0], f0[1], f0[2]) ||
        !amr_inside(S, f0[0] + 5, f0[1] + 5, f0[2] + 5)) {
      atomicOr(status, ST_BAD_ARG);
      continue;
    }
    const long long sy = S.ex[0], sz = (long long)S.ex[0] * S.ex[1];
    const double* q = amr_state(S) + f * S.fs + amr_idx(S, f0[0], f0[1], f0[2]);
    double tmp1[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      double t2[6];
#pragma unroll
      for (int b = 0; b < 6; ++b) {
        const double* r = q + a + b * sy;
        t2[b] = __dadd_rn(__dadd_rn(__dmul_rn(C1, __dadd_rn(r[0], r[5 * sz])), __dmul_rn(C2, __dadd_rn(r[sz], r[4 * sz]))),
                          __dmul_rn(C3, __dadd_rn(r[2 * sz], r[3 * sz])));
      }
      tmp1[a] = __dadd_rn(__dadd_rn(__dmul_rn(C1, __dadd_rn(t2[0], t2[5])), __dmul_rn(C2, __dadd_rn(t2[1], t2[4]))),
                          __dmul_rn(C3, __dadd_rn(t2[2], t2[3])));
    }
    const double v = __dadd_rn(__dadd_rn(__dmul_rn(C1, __dadd_rn(tmp1[0], tmp1[5])), __dmul_rn(C2, __dadd_rn(tmp1[1], tmp1[4]))),
                               __dmul_rn(C3, __dadd_rn(tmp1[2], tmp1[3])));
    const long long od = (long long)f * D.fs + amr_idx(D, c[0], c[1], c[2]);
    if (to_temp) D.K[od] = v;
    else amr_state(D)[od] = v;
  }
}

// Parent state at the child's intermediate time into K (prepare_inter_time_level,
// Parallel.C:4329-4441): average2 (fmisc.f90:1569-1592, 3/8 new + 3/4 old
// - 1/8 older) once the level has two steps behind it, else average
// (fmisc.f90:1532, (new + old)/2), at array point p of block B.
__device__ __forceinline__ void timeinterp_point(const AmrBlock& B, long long p) {
  const int cur = B.lvl[0];
  const double* f1 = B.tl[cur];
  const double* f2 = B.tl[(cur + 2) % 3];
  const double* f3 = B.tl[(cur + 1) % 3];
  if (B.lvl[1] >= 2) {
    const double C1 = 3.0 / 8.0, C2 = 3.0 / 4.0, C3 = -1.0 / 8.0;
    for (int f = 0; f < B.nf; ++f) {
      const long long o = f * B.fs + p;
      B.K[o] = __dadd_rn(__dadd_rn(__dmul_rn(C1, f1[o]), __dmul_rn(C2, f2[o])), __dmul_rn(C3, f3[o]));
    }
  } else {
    for (int f = 0; f < B.nf; ++f) {
      const long long o = f * B.fs + p;
      B.K[o] = __dmul_rn(0.5, __dadd_rn(f1[o], f2[o]));
    }
  }
}

// Over every point of a level's blocks: one thread per block point.
__global__ void k_amr_timeinterp(const AmrBlock* __restrict__ blocks, const int2* __restrict__ tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 tile = tiles[t];
    const AmrBlock& B = blocks[tile.x];
    const long long p = (long long)tile.y + threadIdx.x;
    const long long np = (long long)B.ex[0] * B.ex[1] * B.ex[2];
    if (p >= np) continue;
    timeinterp_point(B, p);
  }
}

// Over boxes of cells (dst = the block; the cells a finer level's
// prolongation reads from it): one thread per box cell.
__global__ void k_amr_timeinterp_boxes(const AmrBlock* __restrict__ blocks, const AmrBox* __restrict__ boxes,
                                       const int2* __restrict__ tiles, int ntiles, unsigned* status) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 tile = tiles[t];
    const AmrBox& bx = boxes[tile.x];
    const int q = tile.y + threadIdx.x;
    if (q >= bx.n[0] * bx.n[1] * bx.n[2]) continue;
    const AmrBlock& B = blocks[bx.dst];
    const int x = bx.lo[0] + q % bx.n[0], y = bx.lo[1] + (q / bx.n[0]) % bx.n[1], z = bx.lo[2] + q / (bx.n[0] * bx.n[1]);
    if (!amr_inside(B, x, y, z)) {
      atomicOr(status, ST_BAD_ARG);
      continue;
    }
    timeinterp_point(B, amr_idx(B, x, y, z));
  }
}

// enforce_ga in place on the current state of every block of a level, as the
// reference does on StateList at the start of each level step
// (bssn_class.C:3052).  One thread per block point.
__global__ void k_amr_enforce(const AmrBlock* __restrict__ blocks, const int2* __restrict__ tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 tile = tiles[t];
    const AmrBlock& B = blocks[tile.x];
    const long long p = (long long)tile.y + threadIdx.x;
    const long long np = (long long)B.ex[0] * B.ex[1] * B.ex[2];
    if (p >= np) continue;
    double* u = B.tl[B.lvl[0]];
    double g[6], a[6];
    for (int m = 0; m < 6; ++m) { g[m] = u[(F_GXX + m) * B.fs + p]; a[m] = u[(F_AXX + m) * B.fs + p]; }
    enforce_ga_point(g, a);
    for (int m = 0; m < 6; ++m) { u[(F_GXX + m) * B.fs + p] = g[m]; u[(F_AXX + m) * B.fs + p] = a[m]; }
  }
}

// Advance a level's time-level ring and step counter.
__global__ void k_amr_rotate(int* lvl) {
  lvl[0] = (lvl[0] + 1) % 3;
  lvl[1] = lvl[1] + 1;
}

}  // namespace amss
