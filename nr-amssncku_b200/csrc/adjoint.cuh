// adjoint.cuh -- vector-Jacobian products of the BSSN RK4 substep (FP64).
//
// The right-hand side of a point is R = P(u(p), D(p)) with D the stencil
// terms of the split form (gradients, Hessians, and "adv" = upwinded advection
// + KO).  Its VJP for output adjoints Rb:
//   1. pointwise: rhs_vjp_bssn (generated from a recording of the kernel's
//      own point function, rhs_vjp_gen.cuh) gives the adjoints of u(p) and of
//      every D slot;
//   2. transpose of the stencils (k_stencil_gather_tiled): the D-slot
//      adjoints of the points whose stencils read a field value are gathered
//      onto it, with the same order / KO / lopsided gates as the forward
//      (blocks without symmetry planes); the upwinded advection also gives
//      the shift its adjoint, Rb * (unweighted upwind derivative)
//      (k_beta_adjoint).
// Outer-face points take the transpose of the Sommerfeld rule instead
// (k_face_vjp, atomicAdd onto the few points it reaches).  The same machinery
// gives the VJP of the Hamiltonian constraint (ham_vjp), the loss integrand of
// the adjoint driver.
#pragma once
#include "rhs_vjp_gen.cuh"

#ifndef AMSS_BETA_UNROLL   // fields per unrolled step of the shift-adjoint loop
#define AMSS_BETA_UNROLL 4
#endif
namespace amss {
constexpr int kBetaUnroll = AMSS_BETA_UNROLL;
}
#ifndef AMSS_ENFVJP_MINB   // resident CTAs per SM the enforce VJP is compiled for
#define AMSS_ENFVJP_MINB 4
#endif
#include "substep_common.cuh"

namespace amss {

// One block as the adjoint kernels see it.
struct AdjBlock {
  BlockView b;
  Coefs<double> C;
  double d2s[3];
  long long npts;
  const double* X;    // linearization point (24 fields, stride b.fs)
  const double* D;    // its stencil terms (slot stride dfs)
  long long dfs;
  const double* Rb;   // adjoint of the right-hand side (24 fields)
  double* Xb;         // += adjoint of X
};

// field of each D slot (Z4c layout, which extends the BSSN one)
struct SlotFieldTable {
  unsigned char f[D_SLOTS_Z4C];
  constexpr SlotFieldTable() : f() {
    for (int F = 0; F < NFIELDS_Z4C; ++F)
      for (int s = doff(F); s < doff(F) + dslots(F); ++s) f[s] = (unsigned char)F;
  }
};
__device__ __forceinline__ int slot_field(int s) {
  constexpr SlotFieldTable t{};
  return t.f[s];
}

// Scatter target of the Sommerfeld transpose: the field value at (i, j, k),
// mirrored cell-centred (with the field's parity) where an index is negative.
struct Scatter {
  const AdjBlock* A;
  __device__ __forceinline__ void add(int F, int i, int j, int k, double v) const {
    const BlockView& b = A->b;
    if (i < 0) { i = -i - 1; if (soa_sign(F, 0) < 0) v = -v; }
    if (j < 0) { j = -j - 1; if (soa_sign(F, 1) < 0) v = -v; }
    if (k < 0) { k = -k - 1; if (soa_sign(F, 2) < 0) v = -v; }
    if (i >= b.ex[0] || j >= b.ex[1] || k >= b.ex[2]) return;   // never read by a gated stencil
    atomicAdd(A->Xb + F * b.fs + i + (long long)j * b.ex[0] + (long long)k * b.ex[0] * b.ex[1], v);
  }
};

// Reads of the generated VJP at one point.
struct VjpIn {
  const AdjBlock* A;
  long long p;
  double hb;   // Hamiltonian-constraint adjoint (ham_vjp), output "field" 99
  __device__ __forceinline__ double c(int F) const { return A->X[F * A->b.fs + p]; }
  __device__ __forceinline__ double d(int s) const { return A->D[s * A->dfs + p]; }
  __device__ __forceinline__ double rb(int F) const { return F == 99 ? hb : A->Rb[F * A->b.fs + p]; }
};

// Writes of the generated VJP: the centre adjoints (each written once, at the
// point) and the D-slot adjoints (stored, then gathered by k_stencil_gather_tiled).
struct VjpStore {
  const AdjBlock* A;
  double* Db;   // D-slot adjoints, same layout as D
  long long p;
  __device__ __forceinline__ void cb(int F, double v) const { A->Xb[F * A->b.fs + p] = v; }
  __device__ __forceinline__ void db(int s, double v) const { Db[s * A->dfs + p] = v; }
};

__device__ __forceinline__ bool on_face_point(const BlockView& b, int i, int j, int k) {
  const int fm = b.face_mask;
  return ((fm & 1) && i == b.ex[0] - 1) || ((fm & 2) && j == b.ex[1] - 1) || ((fm & 4) && k == b.ex[2] - 1) ||
         ((fm & 8) && i == 0) || ((fm & 16) && j == 0) || ((fm & 32) && k == 0);
}

// Pointwise VJP of the right-hand side at the interior (non-face) points:
// centre adjoints into Xb, D-slot adjoints into Db.  Every point's Xb and Db
// are written (zero where the right-hand side does not read the value, and
// everywhere at face points, whose right-hand side is the Sommerfeld rule), so
// neither needs clearing first.
// L2 prefetch (warp 0) of the rows [p0, p0 + 128) of nrows arrays at stride
// `stride` from base: the tile's points only, rounded up to 16 bytes, which
// stays inside rows padded to a multiple of 64 values.
__device__ __forceinline__ void prefetch_tile_rows(const double* base, long long stride, int nrows, long long p0,
                                                   long long npts) {
  if (threadIdx.x >= 32 || p0 >= npts) return;
  const long long nel = npts - p0 < 128 ? npts - p0 : 128;
  const unsigned bytes = (unsigned)((nel * 8 + 15) / 16 * 16);
  for (int r = threadIdx.x; r < nrows; r += 32)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(base + r * stride + p0), "r"(bytes) : "memory");
}

__global__ void __launch_bounds__(128) k_rhs_vjp(const AdjBlock* __restrict__ blocks, double* Db) {
  const AdjBlock& A = blocks[blockIdx.y];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < A.npts;
       p += (long long)gridDim.x * blockDim.x) {
    // this tile's rows meet the point function's one-by-one loads in L2
    const long long p0 = p - threadIdx.x;
    prefetch_tile_rows(A.D, A.dfs, D_SLOTS, p0, A.npts);
    prefetch_tile_rows(A.X, A.b.fs, NFIELDS_BSSN, p0, A.npts);
    prefetch_tile_rows(A.Rb, A.b.fs, NFIELDS_BSSN, p0, A.npts);
    int i, j, k;
    point_ijk(p, A.b.ex, i, j, k);
    if (on_face_point(A.b, i, j, k)) {
      for (int F = 0; F < NFIELDS_BSSN; ++F) A.Xb[F * A.b.fs + p] = 0.0;
      for (int s = 0; s < D_SLOTS; ++s) Db[s * A.dfs + p] = 0.0;
      continue;
    }
    VjpIn in{&A, p, 0.0};
    VjpStore out{&A, Db, p};
    rhs_vjp_bssn<double>(in, out);
#pragma unroll
    for (int F = 0; F < NFIELDS_BSSN; ++F)
      if (!((rhs_vjp_bssn_cb_mask >> F) & 1)) A.Xb[F * A.b.fs + p] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// Transpose of the stencil pass, in gather form.
//
// The stencil pass computes, at every point q, D_s(q) = sum_o w_s(q, o) f(q + o)
// with weights that depend on q only through its gates (derivative order, KO,
// lopsided branch) and, for the advection, on the sign and value of beta(q).
// Its transpose is gathered per target point p:
//   fb(p) = sum_s sum_o Db_s(p - o) w_s(p - o, o),
// so every output point has one owner and no atomics are needed.  The
// offsets are the ones the forward reads: lines o e_d, |o| <= 3 (gradient,
// diagonal Hessian, upwind advection, KO) and planes (oa e_a + ob e_b),
// oa, ob in {-2, -1, 1, 2} (mixed Hessian).  The advection also gives the
// shift an adjoint at p itself: betab_d(p) = sum_f advb_f(p) d12_d u_f,d(p),
// u the unweighted upwind derivative the forward used.  Blocks without
// symmetry planes only (no mirrored reads).

// Upwind weights at offsets -3..3 of the lopsided branches (lopsidediff.f90:
// 321-481): up, centred, and the downwind stencil with the sign the forward
// applies to it.
__device__ __forceinline__ double lop_w(int code, int o) {
  // o is a compile-time constant in every unrolled caller: selects, not a table
  const double up = o == -1 ? -3.0 : o == 0 ? -10.0 : o == 1 ? 18.0 : o == 2 ? -6.0 : o == 3 ? 1.0 : 0.0;
  const double cen = o == -2 ? 1.0 : o == -1 ? -8.0 : o == 1 ? 8.0 : o == 2 ? -1.0 : 0.0;
  const double dn = o == -3 ? -1.0 : o == -2 ? 6.0 : o == -1 ? -18.0 : o == 0 ? 10.0 : o == 1 ? 3.0 : 0.0;
  return code == 0 ? up : code == 1 ? cen : code == 2 ? dn : 0.0;
}
// branch of a point with index x along a direction (lo = imin, hi = imax) for
// a shift component of sign b > 0 / b < 0
__device__ __forceinline__ int lop_code(bool pos, int x, int lo, int hi) {
  if (pos) return x + 3 <= hi ? 0 : (x + 2 <= hi ? 1 : (x + 1 <= hi ? 2 : 3));
  return x - 3 >= lo ? 2 : (x - 2 >= lo ? 1 : (x - 1 >= lo ? 0 : 3));
}

// Per-direction fit flags of one index: bit0 +-2 fits (4th order), bit1 +-1
// fits (2nd order), bit2 +-3 fits (KO), bit3 x <= hi - 1 (lopsided loop).
__device__ __forceinline__ int fit_bits(int x, int hi) {
  return ((x - 2 >= 0 && x + 2 <= hi) ? 1 : 0) | ((x - 1 >= 0 && x + 1 <= hi) ? 2 : 0) |
         ((x - 3 >= 0 && x + 3 <= hi) ? 4 : 0) | ((x <= hi - 1) ? 8 : 0);
}
__device__ __forceinline__ int ord_of(int f) { return (f & 1) ? 2 : ((f & 2) ? 1 : 0); }

// ---------------------------------------------------------------------------
// The transpose as a kernel: one CTA per (x-y tile, field) work item of the
// stencil pass, marching through z like k_deriv.  The in-plane slot adjoints
// of plane m (x/y gradients and Hessians, the mixed Hessians, adv) and the
// shift's x/y components are staged with a 3-cell halo in shared memory by
// cp.async (double-buffered: plane m+1 lands while plane m is used; cells
// outside the block are zero-filled and carry zero weight).  Per plane each
// thread gathers the in-plane terms of its own point (x, y, m) and scatters
// the z-direction terms of its source point (x, y, m) into a register window
// of the outputs at planes m-3 .. m+3; plane m-3 is then complete.  The mixed
// xz / yz terms split into an in-plane gather over x (y) and a z scatter: the
// order gate of the source point q = (x - oa, y, m) is known at plane m, and
// the 2nd-order indicator is F2(q) - F4(q), F2 / F4 the "+-1 / +-2 fit in
// every direction" products.

// In-plane arrays of a field kind: (slot offset within the field, or -1 / -2
// for the shift's x / y component).  Roles: gx gy hxx hyy hxy hxz hyz adv bx by.
template <int KIND>
struct TgMap {
  static constexpr int NA = KIND == 0 ? 10 : (KIND == 1 ? 5 : 3);
  static constexpr int GX = 0, GY = 1, HXX = 2, HYY = 3, HXY = 4, HXZ = 5, HYZ = 6;
  static constexpr int ADV = KIND == 0 ? 7 : (KIND == 1 ? 2 : 0);
  static constexpr int BX = NA - 2, BY = NA - 1;
  __device__ static int src(int a) {
    if (a == BX) return -1;
    if (a == BY) return -2;
    if (KIND == 0) {
      constexpr int k0[8] = {0, 1, 3, 6, 4, 5, 7, 9};
      return k0[a];
    }
    if (KIND == 1) return a == 0 ? 0 : (a == 1 ? 1 : 3);
    return 0;
  }
};
constexpr int kTgPlane = DPLANE;                       // cells of one staged plane (>= (W+6)(H+6))
constexpr size_t kTgSmem = 2 * 10 * kTgPlane * sizeof(double);   // two planes of the widest kind

// The plane cells one thread stages: in-plane offset of each (i + j ex0), or
// -1 outside the block (zero-filled), fixed for the whole march.
struct TgCells {
  int off[DPER];
  __device__ __forceinline__ void init(int x0, int y0, int DSX, int np, int ex0, int ex1) {
#pragma unroll
    for (int e = 0; e < DPER; ++e) {
      const int t = threadIdx.x + e * DTHREADS;
      const int i = x0 - 3 + t % DSX, j = y0 - 3 + t / DSX;
      off[e] = (t < np && i >= 0 && i < ex0 && j >= 0 && j < ex1) ? i + j * ex0 : (t < np ? -1 : -2);
    }
  }
};

template <int KIND>
__device__ __forceinline__ void tg_stage(const AdjBlock& A, const double* Db, int s0, int m, const TgCells& cells,
                                         double* buf) {
  const long long zoff = (long long)m * A.b.ex[0] * A.b.ex[1];
#pragma unroll
  for (int a = 0; a < TgMap<KIND>::NA; ++a) {
    const int sr = TgMap<KIND>::src(a);
    const double* base =
        (sr >= 0 ? Db + (long long)(s0 + sr) * A.dfs : A.X + (long long)(F_BETAX - 1 - sr) * A.b.fs) + zoff;
#pragma unroll
    for (int e = 0; e < DPER; ++e) {
      const int o = cells.off[e];
      if (o >= -1) cp_async8(buf + a * kTgPlane + threadIdx.x + e * DTHREADS, o >= 0 ? base + o : base, o >= 0);
    }
  }
}

// Fit bits (fit_bits) and upwind branch codes (lop_code, b > 0 in bits 0-1,
// b < 0 in bits 2-3) of the points at index x - o, o = -3 .. 3, of one line,
// packed 4 bits per offset; 0 bits (no gate) outside the block.
__device__ __forceinline__ void tg_pack(int x, int hi, unsigned& fits, unsigned& codes) {
  fits = 0u;
  codes = 0u;
#pragma unroll
  for (int o = -3; o <= 3; ++o) {
    const int xq = x - o;
    const bool in = xq >= 0 && xq <= hi;
    const unsigned f = in ? (unsigned)fit_bits(xq, hi) : 0u;
    const unsigned c = in ? (unsigned)(lop_code(true, xq, 0, hi) | (lop_code(false, xq, 0, hi) << 2)) : 15u;
    fits |= f << (4 * (o + 3));
    codes |= c << (4 * (o + 3));
  }
}
__device__ __forceinline__ int tg_bits(unsigned pk, int o) { return (int)((pk >> (4 * (o + 3))) & 15u); }

// L2 prefetch, one 128-byte line per thread and step, of plane m's tile rows
// (with halo) of every array the march reads, a few planes before it is staged.
template <int KIND>
__device__ __forceinline__ void tg_prefetch(const AdjBlock& A, const double* Db, int s0, int m, int x0, int y0,
                                            int W, int H) {
  const BlockView& b = A.b;
  const int ex0 = b.ex[0], ex1 = b.ex[1];
  const int xl = x0 - 3 < 0 ? 0 : x0 - 3, xh = x0 + W + 3 > ex0 ? ex0 : x0 + W + 3;
  const int yl = y0 - 3 < 0 ? 0 : y0 - 3, yh = y0 + H + 3 > ex1 ? ex1 : y0 + H + 3;
  const int lpr = ((xh - xl) * 8 + 127) / 128, nr = yh - yl;
  const int na = TgMap<KIND>::NA + (KIND == 0 ? 3 : (KIND == 1 ? 2 : 1));   // + the z-column arrays
  const long long zoff = (long long)m * ex0 * ex1 + xl;
  for (int t = threadIdx.x; t < na * nr * lpr; t += DTHREADS) {
    const int a = t / (nr * lpr), rem = t - a * nr * lpr, r = rem / lpr, c = rem - r * lpr;
    const double* base;
    if (a < TgMap<KIND>::NA) {
      const int sr = TgMap<KIND>::src(a);
      base = sr >= 0 ? Db + (long long)(s0 + sr) * A.dfs : A.X + (long long)(F_BETAX - 1 - sr) * b.fs;
    } else {
      const int z = a - TgMap<KIND>::NA;   // beta^z, then gz and hzz as the kind has them
      base = z == 0 ? A.X + (long long)F_BETAZ * b.fs : Db + (long long)(s0 + (z == 1 ? 2 : 8)) * A.dfs;
    }
    const char* row = (const char*)(base + zoff + (long long)(yl + r) * ex0);
    const int off = c * 128 < (xh - xl - 1) * 8 ? c * 128 : (xh - xl - 1) * 8;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(row + off));
  }
}

template <int KIND>
__device__ __forceinline__ void tg_column(const AdjBlock& A, const double* __restrict__ Db, int F, int x0, int y0,
                                          double* smem) {
  using M = TgMap<KIND>;
  const BlockView& b = A.b;
  const Coef<double>& C = A.C.t;
  const int ex0 = b.ex[0], ex1 = b.ex[1], ex2 = b.ex[2];
  const int hix = ex0 - 1, hiy = ex1 - 1, hiz = ex2 - 1;
  const int W = deriv_tile_w(ex0), H = DTHREADS / W;
  const int DSX = W + 6, np = DSX * (H + 6);
  const int li = threadIdx.x % W, lj = threadIdx.x / W;
  const int x = x0 + li, y = y0 + lj;
  const bool mine = lj < H && x < ex0 && y < ex1;
  const int own = (lj < H ? lj + 3 : 3) * DSX + (li + 3);
  const int s0 = doff(F);
  const int fbx = fit_bits(x, hix), fby = fit_bits(y, hiy);
  unsigned pfx, pcx, pfy, pcy;
  tg_pack(x, hix, pfx, pcx);
  tg_pack(y, hiy, pfy, pcy);
  const long long sz = (long long)ex0 * ex1;
  const long long pxy = mine ? x + (long long)y * ex0 : 0;
  const double* gzc = Db + (long long)(s0 + 2) * A.dfs + pxy;
  const double* hzc = Db + (long long)(s0 + 8) * A.dfs + pxy;
  const double* bzc = A.X + (long long)F_BETAZ * b.fs + pxy;
  double* out = A.Xb + (long long)F * b.fs + pxy;
  double acc[7];
#pragma unroll
  for (int t = 0; t < 7; ++t) acc[t] = 0.0;
  const double w4[5] = {1.0, -8.0, 0.0, 8.0, -1.0};   // offsets -2..2

  TgCells cells;
  cells.init(x0, y0, DSX, np, ex0, ex1);
  tg_stage<KIND>(A, Db, s0, 0, cells, smem);
  cp_async_commit();
#pragma unroll 1
  for (int m = 0; m < ex2 + 3; ++m) {
    if (m < ex2) {
      if (m + 1 < ex2) tg_stage<KIND>(A, Db, s0, m + 1, cells, smem + ((m + 1) & 1) * 10 * kTgPlane);
      cp_async_commit();
      if (m + 5 < ex2) tg_prefetch<KIND>(A, Db, s0, m + 5, x0, y0, W, H);
      double gz = 0.0, hzz = 0.0, bz = 0.0;
      if (mine) {
        if (KIND != 2) gz = __ldg(gzc + m * sz);
        if (KIND == 0) hzz = __ldg(hzc + m * sz);
        bz = __ldg(bzc + m * sz);
      }
      cp_async_wait<1>();
      __syncthreads();
      const double* P = smem + (m & 1) * 10 * kTgPlane;
      if (mine) {
        const int fbz = fit_bits(m, hiz);
        double ip = 0.0;
        // x and y lines through (x, y, m); cells outside the block are zero in P
#pragma unroll
        for (int d = 0; d < 2; ++d) {
          const unsigned pf = d == 0 ? pfx : pfy, pc = d == 0 ? pcx : pcy;
          const int st = d == 0 ? 1 : DSX;
          const int other = (d == 0 ? fby : fbx) & fbz;
          const double kod = C.ko / C.h[d], lpd = C.d12[d];
#pragma unroll
          for (int o = -3; o <= 3; ++o) {
            const int f = other & tg_bits(pf, o);
            const int c = own - o * st;
            if (KIND != 2 && o >= -2 && o <= 2) {
              const int ord = ord_of(f);
              if (o != 0) {
                const double wg = ord == 2 ? C.d12[d] * w4[o + 2] : (ord == 1 && (o == 1 || o == -1) ? C.d2[d] * o : 0.0);
                ip += P[(d == 0 ? M::GX : M::GY) * kTgPlane + c] * wg;
              }
              if (KIND == 0) {
                const double h4 = o == 0 ? -30.0 : (o == -1 || o == 1) ? 16.0 : -1.0;
                const double wh = ord == 2 ? C.Fdd[d] * h4
                                           : (ord == 1 && o >= -1 && o <= 1 ? C.Sdd[d] * (o == 0 ? -2.0 : 1.0) : 0.0);
                ip += P[(d == 0 ? M::HXX : M::HYY) * kTgPlane + c] * wh;
              }
            }
            const double ab = P[M::ADV * kTgPlane + c];
            const double wko = o == 0 ? -20.0 : (o == 1 || o == -1) ? 15.0 : (o == 2 || o == -2) ? -6.0 : 1.0;
            double w = (f & 4) ? kod * wko : 0.0;
            if (f & 8) {
              const double bq = P[(d == 0 ? M::BX : M::BY) * kTgPlane + c];
              const int cq = tg_bits(pc, o);
              w += bq * lpd * lop_w(bq > 0.0 ? (cq & 3) : (cq >> 2), o);
            }
            ip += ab * w;
          }
        }
        if (KIND == 0) {
          // xy cross stencil, gathered in the plane
#pragma unroll
          for (int oa = -2; oa <= 2; ++oa) {
            if (oa == 0) continue;
            const int fa = tg_bits(pfx, oa) & fbz;
#pragma unroll
            for (int ob = -2; ob <= 2; ++ob) {
              if (ob == 0) continue;
              const int ord = ord_of(fa & tg_bits(pfy, ob));
              const double w = ord == 2 ? C.Fxy * w4[oa + 2] * w4[ob + 2]
                                        : (ord == 1 && oa * oa == 1 && ob * ob == 1 ? C.Sxy * (double)(oa * ob) : 0.0);
              ip += P[M::HXY * kTgPlane + own - oa - ob * DSX] * w;
            }
          }
        }
        acc[3] += ip;
        // z-direction terms of the source point (x, y, m), scattered to planes m-3 .. m+3
        const int fq = fbx & fby & fbz;
        const int ordq = ord_of(fq);
        if (KIND != 2) {
#pragma unroll
          for (int o = -2; o <= 2; ++o) {
            if (o == 0) continue;
            acc[3 + o] += gz * (ordq == 2 ? C.d12[2] * w4[o + 2] : (ordq == 1 && (o == 1 || o == -1) ? C.d2[2] * o : 0.0));
          }
        }
        if (KIND == 0) {
#pragma unroll
          for (int o = -2; o <= 2; ++o) {
            const double h4 = o == 0 ? -30.0 : (o == -1 || o == 1) ? 16.0 : -1.0;
            acc[3 + o] += hzz * (ordq == 2 ? C.Fdd[2] * h4
                                           : (ordq == 1 && o >= -1 && o <= 1 ? C.Sdd[2] * (o == 0 ? -2.0 : 1.0) : 0.0));
          }
          // xz and yz: in-plane gather along x (y) of the source points q = (x - oa, y, m), then z scatter
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const unsigned pf = e == 0 ? pfx : pfy;
            const int st = e == 0 ? 1 : DSX;
            const int other = (e == 0 ? fby : fbx) & fbz;
            const int arr = e == 0 ? M::HXZ : M::HYZ;
            double g4 = 0.0, g1 = 0.0;
#pragma unroll
            for (int oa = -2; oa <= 2; ++oa) {
              if (oa == 0) continue;
              const int f = other & tg_bits(pf, oa);
              const double v = P[arr * kTgPlane + own - oa * st];
              if (f & 1) g4 += w4[oa + 2] * v;
              if ((oa == 1 || oa == -1) && (f & 2) && !(f & 1)) g1 += (double)oa * v;
            }
            const double F4 = e == 0 ? C.Fxz : C.Fyz, S2 = e == 0 ? C.Sxz : C.Syz;
#pragma unroll
            for (int oc = -2; oc <= 2; ++oc) {
              if (oc == 0) continue;
              double w = F4 * w4[oc + 2] * g4;
              if (oc == 1 || oc == -1) w += S2 * (double)oc * g1;
              acc[3 + oc] += w;
            }
          }
        }
        // adv along z: KO and the upwind stencil of the source point
        {
          const double ab = P[M::ADV * kTgPlane + own];
          const int code = (fq & 8) && bz != 0.0 ? lop_code(bz > 0.0, m, 0, hiz) : 3;
          const double kod = (fq & 4) ? C.ko / C.h[2] : 0.0;
          const double lz = bz * C.d12[2];
#pragma unroll
          for (int o = -3; o <= 3; ++o) {
            const double wko = o == 0 ? -20.0 : (o == 1 || o == -1) ? 15.0 : (o == 2 || o == -2) ? -6.0 : 1.0;
            acc[3 + o] += ab * (kod * wko + lz * lop_w(code, o));
          }
        }
      }
      __syncthreads();   // every thread is done with plane m's buffer before plane m+2 is staged into it
    }
    const int k = m - 3;
    if (k >= 0 && mine) out[k * sz] += acc[0];
#pragma unroll
    for (int t = 0; t < 6; ++t) acc[t] = acc[t + 1];
    acc[6] = 0.0;
  }
  cp_async_wait<0>();
}

// Xb += transpose(stencil pass)(Db), one CTA per (tile, field) item of the
// stencil pass's work list (BSSN layout, no symmetry planes).
__global__ void __launch_bounds__(DTHREADS, 2) k_stencil_gather_tiled(const AdjBlock* __restrict__ A,
                                                                      const DerivItem* __restrict__ items,
                                                                      const double* __restrict__ Db) {
  extern __shared__ __align__(16) unsigned char tg_smem[];
  const DerivItem it = items[blockIdx.x];
  double* smem = reinterpret_cast<double*>(tg_smem);
  switch (dkind(it.field)) {
    case 0: tg_column<0>(*A, Db, it.field, it.x0, it.y0, smem); break;
    case 1: tg_column<1>(*A, Db, it.field, it.x0, it.y0, smem); break;
    default: tg_column<2>(*A, Db, it.field, it.x0, it.y0, smem); break;
  }
}

// The shift as the advecting velocity: betab_d(p) += sum_F advb_F(p) d12_d
// sum_o w_o f_F(p + o e_d), w the upwind weights the forward used at p
// (lopsidediff.f90:321-481).
__global__ void __launch_bounds__(128) k_beta_adjoint(const AdjBlock* __restrict__ A, const double* __restrict__ Db) {
  const BlockView& b = A->b;
  const Coef<double>& C = A->C.t;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < A->npts;
       p += (long long)gridDim.x * blockDim.x) {
    int id[3];
    point_ijk(p, b.ex, id[0], id[1], id[2]);
    const long long str[3] = {1, b.ex[0], (long long)b.ex[0] * b.ex[1]};
    // face points (no advection term, zero adv adjoint) are skipped: every
    // other point's upwind stencil lies inside the block
    if (on_face_point(b, id[0], id[1], id[2])) continue;
    if (!(fit_bits(id[0], b.ex[0] - 1) & fit_bits(id[1], b.ex[1] - 1) & fit_bits(id[2], b.ex[2] - 1) & 8)) continue;
    int code[3];
    bool any = false;
    for (int d = 0; d < 3; ++d) {
      const double bq = A->X[(F_BETAX + d) * b.fs + p];
      code[d] = bq == 0.0 ? 3 : lop_code(bq > 0.0, id[d], 0, b.ex[d] - 1);
      any = any || code[d] != 3;
    }
    if (!any) continue;
    // per direction: the five points of the upwind stencil the forward used and
    // their weights (all zero where it added nothing), so the field loop has no
    // branches and its loads can be issued together
    long long o0[3], st[3];
    double w[3][5];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int c = code[d];
      st[d] = c == 3 ? 0 : str[d];
      o0[d] = c == 0 ? -1 : (c == 1 ? -2 : -3);
#pragma unroll
      for (int t = 0; t < 5; ++t) w[d][t] = c == 3 ? 0.0 : lop_w(c, (int)o0[d] + t);
    }
    double bb[3] = {0.0, 0.0, 0.0};
#pragma unroll kBetaUnroll
    for (int F = 0; F < NFIELDS_BSSN; ++F) {
      const double ab = Db[(doff(F) + dslots(F) - 1) * A->dfs + p];
      const double* X = A->X + F * b.fs + p;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double u = 0.0;
#pragma unroll
        for (int t = 0; t < 5; ++t) u += w[d][t] * X[(o0[d] + t) * st[d]];
        bb[d] += ab * C.d12[d] * u;
      }
    }
    for (int d = 0; d < 3; ++d) A->Xb[(F_BETAX + d) * b.fs + p] += bb[d];
  }
}

// Transpose of the Sommerfeld rule (sommerfeld_rout.f90:378-440) at the
// outer-face points of a level-0 block.
__global__ void __launch_bounds__(128) k_face_vjp(const AdjBlock* __restrict__ blocks, const int2* __restrict__ faces,
                                                  int nfaces) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nfaces; t += gridDim.x * blockDim.x) {
    const AdjBlock& A = blocks[faces[t].x];
    const long long p = faces[t].y;
    int i, j, k;
    point_ijk(p, A.b.ex, i, j, k);
    const Scatter S{&A};
    const double x = A.b.X[i], y = A.b.Y[j], z = A.b.Z[k];
    const double R = sqrt(x * x + y * y + z * z);
    const double pos[3] = {x, y, z};
    const int id[3] = {i, j, k};
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      lo[d] = ((A.b.lowsym_mask >> d) & 1) ? -1 : 0;
      hi[d] = A.b.ex[d] - 1;
    }
    for (int F = 0; F < NFIELDS_BSSN; ++F) {
      const double v = (F == F_CHI || F == F_TRK || F == F_LAP) ? 1.4142135623730951 : 1.0;
      const double rb = A.Rb[F * A.b.fs + p];
      if (rb == 0.0) continue;
      const double g = -v / R * rb;   // d rhs / d (fd_d x_d + f0)
      S.add(F, i, j, k, g);
      for (int d = 0; d < 3; ++d) {
        const double wv = v * pos[d] / R;
        if (wv == 0.0) continue;
        const double c = g * pos[d] * A.d2s[d];
        auto at = [&](int o, double w) {
          S.add(F, i + (d == 0 ? o : 0), j + (d == 1 ? o : 0), k + (d == 2 ? o : 0), c * w);
        };
        if (wv > 0) {
          if (id[d] - 2 >= lo[d]) { at(0, 3); at(-1, -4); at(-2, 1); }
          else if (id[d] - 1 >= lo[d]) { at(-1, -1); at(1, 1); }
          else { at(2, -1); at(1, 4); at(0, -3); }
        } else {
          if (id[d] + 2 <= hi[d]) { at(2, -1); at(1, 4); at(0, -3); }
          else if (id[d] + 1 <= hi[d]) { at(-1, -1); at(1, 1); }
          else { at(0, 3); at(-1, -4); at(-2, 1); }
        }
      }
    }
  }
}

// Hamiltonian constraint of the interior cells [gw, ex - gw) of a block:
// H written to Hout, sum H^2 dV added to *loss.
__global__ void __launch_bounds__(128) k_ham_loss(const AdjBlock* __restrict__ blocks, int gw, double dV,
                                                  double* Hout, double* loss) {
  const AdjBlock& A = blocks[blockIdx.y];
  double acc = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < A.npts;
       p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    point_ijk(p, A.b.ex, i, j, k);
    double h = 0.0;
    if (i >= gw && j >= gw && k >= gw && i < A.b.ex[0] - gw && j < A.b.ex[1] - gw && k < A.b.ex[2] - gw) {
      VjpIn in{&A, p, 0.0};
      h = ham_fwd<double>(in);
      acc += h * h * dV;
    }
    Hout[p] = h;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// Pointwise VJP of sum H^2 dV (Hb = 2 H dV on the interior cells): centre
// adjoints into Xb, D-slot adjoints into Db (gathered by k_stencil_gather_tiled).
__global__ void __launch_bounds__(128) k_ham_vjp(const AdjBlock* __restrict__ blocks, int gw, double dV,
                                                 const double* H, double* Db) {
  const AdjBlock& A = blocks[blockIdx.y];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < A.npts;
       p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    point_ijk(p, A.b.ex, i, j, k);
    if (!(i >= gw && j >= gw && k >= gw && i < A.b.ex[0] - gw && j < A.b.ex[1] - gw && k < A.b.ex[2] - gw))
      continue;
    VjpIn in{&A, p, 2.0 * H[p] * dV};
    VjpStore out{&A, Db, p};
    ham_vjp<double>(in, out);
  }
}

// enforce_ga_point's VJP: adjoint of the metric / A~ components of Z (pre-
// enforce values, offsets) given the adjoint of E(Z); other fields pass through.
// enforce_vjp's reads: the pre-enforce metric / A~ (Z) and the adjoint of
// E(Z), given as the sum of up to two arrays.
struct EnfIn {
  const double* Z;
  const double* E1;
  const double* E2;
  long long fs, p;
  __device__ __forceinline__ double c(int m) const { return Z[(F_GXX + m) * fs + p]; }
  __device__ __forceinline__ double d(int) const { return 0.0; }
  __device__ __forceinline__ double rb(int m) const {
    const long long o = (F_GXX + m) * fs + p;
    return E2 ? E1[o] + E2[o] : E1[o];
  }
};
struct EnfOut {
  double zb[12];
  __device__ __forceinline__ void cb(int m, double v) { zb[m] = v; }
  __device__ __forceinline__ void db(int, double) {}
};

// The reverse of one enforce + chi floor, fused with what consumes its
// result: Zb = mask(Z) E'(Z)^T (E1 + E2) per point (chi masked where the floor
// held Z at chitiny; E2 may be null), then
//   out = Zb (if out), acc0 += Zb (if acc0), acc1 += c1 Zb (if acc1).
// ACC: acc0 += Zb, acc1 += c1 Zb (a substep's reverse); else out = Zb with
// E2 added to E1 (the step start).  No two arrays alias.
template <bool ACC>
__global__ void __launch_bounds__(128, AMSS_ENFVJP_MINB) k_enforce_vjp(const double* __restrict__ Z, const double* __restrict__ E1,
                                                     const double* __restrict__ E2, double* __restrict__ out,
                                                     double* __restrict__ acc0, double* __restrict__ acc1,
                                                     double c1, long long n, long long fs, double chitiny) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    EnfIn in{Z, E1, ACC ? nullptr : E2, fs, p};
    EnfOut eo;
    enforce_vjp<double>(in, eo);
    const bool floor_held = Z[F_CHI * fs + p] == chitiny;
#pragma unroll
    for (int f = 0; f < NFIELDS_BSSN; ++f) {
      const long long o = f * fs + p;
      double v;
      if (f >= F_GXX && f <= F_AZZ) v = eo.zb[f - F_GXX];
      else v = ACC ? E1[o] : E1[o] + E2[o];
      if (f == F_CHI && floor_held) v = 0.0;
      if (ACC) {
        acc0[o] += v;
        acc1[o] += c1 * v;
      } else {
        out[o] = v;
      }
    }
  }
}

// Seed of one step's reverse: with Yb = mask(U_new) Ub,
//   U0b = Yb, R3b = R0b = dt/6 Yb, R1b = R2b = dt/3 Yb.
__global__ void __launch_bounds__(128) k_step_seed(const double* __restrict__ Ub, const double* __restrict__ Unew,
                                                   double* U0b, double* R0b, double* R1b, double* R2b, double* R3b,
                                                   double dt, long long n, long long fs, double chitiny) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const bool floor_held = Unew[F_CHI * fs + p] == chitiny;
#pragma unroll 4
    for (int f = 0; f < NFIELDS_BSSN; ++f) {
      const long long o = f * fs + p;
      const double y = (f == F_CHI && floor_held) ? 0.0 : Ub[o];
      U0b[o] = y;
      R0b[o] = (dt / 6.0) * y;
      R3b[o] = (dt / 6.0) * y;
      R1b[o] = (dt / 3.0) * y;
      R2b[o] = (dt / 3.0) * y;
    }
  }
}

}  // namespace amss
