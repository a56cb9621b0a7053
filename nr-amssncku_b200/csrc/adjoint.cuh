// adjoint.cuh -- vector-Jacobian products of the BSSN RK4 substep (FP64).
//
// The right-hand side of a point is R = P(u(p), D(p)) with D the stencil
// terms of the split form (gradients, Hessians, and "adv" = upwinded advection
// + KO).  Its VJP for output adjoints Rb:
//   1. pointwise: rhs_vjp_bssn (generated from a recording of the kernel's
//      own point function, rhs_vjp_gen.cuh) gives the adjoints of u(p) and of
//      every D slot;
//   2. transpose of the stencils: each D-slot adjoint is scattered back onto
//      the field values its stencil read, with the same order / KO / lopsided
//      gates and the same mirroring of negative indices (parity of the field)
//      as the forward; the upwinded advection also gives the shift its
//      adjoint, Rb * (unweighted upwind derivative).
// Outer-face points take the transpose of the Sommerfeld rule instead.  All
// contributions are accumulated with atomicAdd into the adjoint of the stage
// input.  The same machinery gives the VJP of the Hamiltonian constraint
// (ham_vjp), the loss integrand of the adjoint driver.
#pragma once
#include "rhs_vjp_gen.cuh"
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

// Scatter target: the field value at (i, j, k), mirrored cell-centred (with the
// field's parity) where an index is negative, as the forward's padded reads.
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
  __device__ __forceinline__ double get(int F, int i, int j, int k) const {
    const BlockView& b = A->b;
    bool neg = false;
    if (i < 0) { i = -i - 1; neg ^= soa_sign(F, 0) < 0; }
    if (j < 0) { j = -j - 1; neg ^= soa_sign(F, 1) < 0; }
    if (k < 0) { k = -k - 1; neg ^= soa_sign(F, 2) < 0; }
    const double v = A->X[F * b.fs + i + (long long)j * b.ex[0] + (long long)k * b.ex[0] * b.ex[1]];
    return neg ? -v : v;
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
// point) and the D-slot adjoints (stored, then gathered by k_stencil_gather).
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
__global__ void __launch_bounds__(128) k_rhs_vjp(const AdjBlock* __restrict__ blocks, double* Db) {
  const AdjBlock& A = blocks[blockIdx.y];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < A.npts;
       p += (long long)gridDim.x * blockDim.x) {
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
// so every thread owns its output point and no atomics are needed.  The
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

struct GatherPt {
  const AdjBlock* A;
  const double* Db;   // slot 0 at this point: slot s at Db[s * dfs], neighbours at int offsets
  const double* beta; // beta^x at this point (field stride fs)
  int dfs, fs;
  int id[3];
  int str[3];
  int fb[3];   // fit bits of p's own indices
  __device__ __forceinline__ double db(int s, int off) const { return __ldg(Db + s * dfs + off); }
};

// Contribution to fb(p) of every slot of field F (KIND: 0 gradient + Hessian
// + adv, 1 gradient + adv, 2 adv only); slot base `s0`.  FAST: p is at least 6
// cells from every face, so every point its transpose reads has full gates.
template <int KIND, bool FAST>
__device__ __forceinline__ double gather_field(const GatherPt& g, int s0) {
  const Coef<double>& C = g.A->C.t;
  const BlockView& b = g.A->b;
  const int nsl = KIND == 0 ? 10 : (KIND == 1 ? 4 : 1);
  const int sadv = s0 + nsl - 1;
  double acc = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int d1 = d == 0 ? 1 : 0, d2 = d == 2 ? 1 : 2;
    const int other = FAST ? 15 : (g.fb[d1] & g.fb[d2]);
    const int hi = b.ex[d] - 1;
    const double kod = C.ko / C.h[d], lpd = C.d12[d];
#pragma unroll
    for (int o = -3; o <= 3; ++o) {
      const int x = g.id[d] - o;
      if (!FAST && (x < 0 || x > hi)) continue;
      const int q = -o * g.str[d];
      const int f = FAST ? 15 : (other & fit_bits(x, hi));
      if (KIND != 2 && o >= -2 && o <= 2) {
        const int ord = FAST ? 2 : ord_of(f);
        const double w4 = o == -2 ? 1.0 : o == -1 ? -8.0 : o == 1 ? 8.0 : o == 2 ? -1.0 : 0.0;
        const double w2 = o == -1 ? -1.0 : o == 1 ? 1.0 : 0.0;
        if (o != 0) {
          const double wg = ord == 2 ? C.d12[d] * w4 : (ord == 1 ? C.d2[d] * w2 : 0.0);
          acc += g.db(s0 + d, q) * wg;
        }
        if (KIND == 0) {
          const double h4 = o == 0 ? -30.0 : (o == -1 || o == 1) ? 16.0 : -1.0;
          const double h2 = o == 0 ? -2.0 : (o == -1 || o == 1) ? 1.0 : 0.0;
          const int sh = s0 + 3 + (d == 0 ? 0 : d == 1 ? 3 : 5);   // xx, yy, zz
          if (FAST || ord == 2) acc += g.db(sh, q) * (C.Fdd[d] * h4);
          else if (ord == 1 && o >= -1 && o <= 1) acc += g.db(sh, q) * (C.Sdd[d] * h2);
        }
      }
      const double ab = g.db(sadv, q);
      const double wko = o == 0 ? -20.0 : (o == 1 || o == -1) ? 15.0 : (o == 2 || o == -2) ? -6.0 : 1.0;
      double w = (f & 4) ? kod * wko : 0.0;
      if (f & 8) {
        const double bq = __ldg(g.beta + d * g.fs + q);
        const int code = FAST ? (bq > 0.0 ? 0 : 2) : lop_code(bq > 0.0, x, 0, hi);
        w += bq * lpd * lop_w(code, o);   // zero where beta vanishes
      }
      acc += ab * w;
    }
  }
  if (KIND == 0) {
#pragma unroll
    for (int m = 0; m < 3; ++m) {   // xy, xz, yz
      const int a = m == 2 ? 1 : 0, c = m == 0 ? 1 : 2, e = 3 - a - c;
      const int sm = s0 + 3 + (m == 0 ? 1 : m == 1 ? 2 : 4);
      const double F4 = m == 0 ? C.Fxy : m == 1 ? C.Fxz : C.Fyz;
      const double S2 = m == 0 ? C.Sxy : m == 1 ? C.Sxz : C.Syz;
      const int ha = b.ex[a] - 1, hc = b.ex[c] - 1;
#pragma unroll
      for (int oa = -2; oa <= 2; ++oa) {
        if (oa == 0) continue;
        const int xa = g.id[a] - oa;
        if (!FAST && (xa < 0 || xa > ha)) continue;
        const int fa = FAST ? 15 : (fit_bits(xa, ha) & g.fb[e]);
        const double wa = oa == -2 ? 1.0 : oa == -1 ? -8.0 : oa == 1 ? 8.0 : -1.0;
        double row = 0.0;   // FAST: the 4th-order taps of this oa summed over oc first
#pragma unroll
        for (int oc = -2; oc <= 2; ++oc) {
          if (oc == 0) continue;
          const int xc = g.id[c] - oc;
          if (!FAST && (xc < 0 || xc > hc)) continue;
          const double wc = oc == -2 ? 1.0 : oc == -1 ? -8.0 : oc == 1 ? 8.0 : -1.0;
          const double v = g.db(sm, -oa * g.str[a] - oc * g.str[c]);
          if (FAST) {
            row += wc * v;
          } else {
            const int ord = ord_of(fa & fit_bits(xc, hc));
            if (ord == 2) acc += v * (F4 * wa * wc);
            else if (ord == 1 && oa * oa == 1 && oc * oc == 1) acc += v * (S2 * (double)(oa * oc));
          }
        }
        if (FAST) acc += row * (F4 * wa);
      }
    }
  }
  return acc;
}

// Xb_F += transpose(stencil pass)(Db) of field F = blockIdx.y at every point
// (BSSN layout, 135 slots); one thread per (point, field).  Offsets are 32-bit
// (amss_adjoint_create bounds D_SLOTS x the field stride).
__global__ void __launch_bounds__(128) k_stencil_gather(const AdjBlock* __restrict__ A, const double* __restrict__ Db) {
  const BlockView& b = A->b;
  const int F = blockIdx.y;
  const int s0 = doff(F), n = dslots(F);
  const int npts = (int)A->npts;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npts; p += gridDim.x * blockDim.x) {
    GatherPt g;
    g.A = A;
    g.Db = Db + p;
    g.beta = A->X + F_BETAX * b.fs + p;
    g.dfs = (int)A->dfs;
    g.fs = (int)b.fs;
    g.id[0] = p % b.ex[0];
    g.id[1] = (p / b.ex[0]) % b.ex[1];
    g.id[2] = p / (b.ex[0] * b.ex[1]);
    g.str[0] = 1;
    g.str[1] = b.ex[0];
    g.str[2] = b.ex[0] * b.ex[1];
    bool fast = true;
    for (int d = 0; d < 3; ++d) {
      g.fb[d] = fit_bits(g.id[d], b.ex[d] - 1);
      fast = fast && g.id[d] >= 6 && g.id[d] <= b.ex[d] - 7;
    }
    double acc;
    if (n == 10) acc = fast ? gather_field<0, true>(g, s0) : gather_field<0, false>(g, s0);
    else if (n == 4) acc = fast ? gather_field<1, true>(g, s0) : gather_field<1, false>(g, s0);
    else acc = fast ? gather_field<2, true>(g, s0) : gather_field<2, false>(g, s0);
    A->Xb[F * b.fs + p] += acc;
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
    if (!(fit_bits(id[0], b.ex[0] - 1) & fit_bits(id[1], b.ex[1] - 1) & fit_bits(id[2], b.ex[2] - 1) & 8)) continue;
    int code[3];
    bool any = false;
    for (int d = 0; d < 3; ++d) {
      const double bq = A->X[(F_BETAX + d) * b.fs + p];
      code[d] = bq == 0.0 ? 3 : lop_code(bq > 0.0, id[d], 0, b.ex[d] - 1);
      any = any || code[d] != 3;
    }
    if (!any) continue;
    double bb[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
    for (int F = 0; F < NFIELDS_BSSN; ++F) {
      const double ab = Db[(doff(F) + dslots(F) - 1) * A->dfs + p];
      if (ab == 0.0) continue;
      const double* X = A->X + F * b.fs + p;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (code[d] == 3) continue;
        double u = 0.0;
#pragma unroll
        for (int o = -3; o <= 3; ++o) {
          const double w = lop_w(code[d], o);
          if (w != 0.0) u += w * X[o * str[d]];
        }
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
// adjoints into Xb, D-slot adjoints into Db (gathered by k_stencil_gather).
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
__global__ void __launch_bounds__(128) k_enforce_vjp(const double* __restrict__ Z, const double* E1,
                                                     const double* E2, double* out, double* acc0, double* acc1,
                                                     double c1, long long n, long long fs, double chitiny) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    EnfIn in{Z, E1, E2, fs, p};
    EnfOut eo;
    enforce_vjp<double>(in, eo);
    const bool floor_held = Z[F_CHI * fs + p] == chitiny;
#pragma unroll
    for (int f = 0; f < NFIELDS_BSSN; ++f) {
      const long long o = f * fs + p;
      double v;
      if (f >= F_GXX && f <= F_AZZ) v = eo.zb[f - F_GXX];
      else v = E2 ? E1[o] + E2[o] : E1[o];
      if (f == F_CHI && floor_held) v = 0.0;
      if (out) out[o] = v;
      if (acc0) acc0[o] += v;
      if (acc1) acc1[o] += c1 * v;
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
