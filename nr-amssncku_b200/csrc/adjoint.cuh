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

// Writes of the generated VJP: the centre adjoint, and every D-slot adjoint
// through the transpose of its stencil.
struct VjpOut {
  const AdjBlock* A;
  long long p;
  int i, j, k;
  PointGates G;
  Scatter S;

  __device__ __forceinline__ void cb(int F, double v) const { S.add(F, i, j, k, v); }

  __device__ __forceinline__ void line(int F, int d, int o, double v) const {
    S.add(F, i + (d == 0 ? o : 0), j + (d == 1 ? o : 0), k + (d == 2 ? o : 0), v);
  }
  __device__ __forceinline__ void plane(int F, int da, int oa, int db, int ob, double v) const {
    int ii = i, jj = j, kk = k;
    (da == 0 ? ii : da == 1 ? jj : kk) += oa;
    (db == 0 ? ii : db == 1 ? jj : kk) += ob;
    S.add(F, ii, jj, kk, v);
  }

  // fderivs (diff_new.f90:946-1104)
  __device__ __forceinline__ void grad(int F, int d, double v) const {
    const Coef<double>& C = A->C.t;
    if (G.ord == 2) {
      const double c = C.d12[d] * v;
      line(F, d, -2, c); line(F, d, -1, -8.0 * c); line(F, d, 1, 8.0 * c); line(F, d, 2, -c);
    } else if (G.ord == 1) {
      const double c = C.d2[d] * v;
      line(F, d, -1, -c); line(F, d, 1, c);
    }
  }
  // fdderivs (diff_new.f90:1338-1528); m: xx xy xz yy yz zz
  __device__ __forceinline__ void hess(int F, int m, double v) const {
    const Coef<double>& C = A->C.t;
    const int da[6] = {0, 0, 0, 1, 1, 2}, db[6] = {0, 1, 2, 1, 2, 2};
    const int a = da[m], b = db[m];
    if (a == b) {
      if (G.ord == 2) {
        const double c = C.Fdd[a] * v;
        line(F, a, -2, -c); line(F, a, -1, 16.0 * c); line(F, a, 0, -30.0 * c);
        line(F, a, 1, 16.0 * c); line(F, a, 2, -c);
      } else if (G.ord == 1) {
        const double c = C.Sdd[a] * v;
        line(F, a, -1, c); line(F, a, 0, -2.0 * c); line(F, a, 1, c);
      }
    } else {
      if (G.ord == 2) {
        const double cf = (m == 1 ? C.Fxy : m == 2 ? C.Fxz : C.Fyz) * v;
        const int o[4] = {-2, -1, 1, 2};
        const double w[4] = {1.0, -8.0, 8.0, -1.0};
        for (int x = 0; x < 4; ++x)
          for (int y = 0; y < 4; ++y) plane(F, a, o[x], b, o[y], cf * w[x] * w[y]);
      } else if (G.ord == 1) {
        const double cf = (m == 1 ? C.Sxy : m == 2 ? C.Sxz : C.Syz) * v;
        plane(F, a, -1, b, -1, cf); plane(F, a, 1, b, -1, -cf);
        plane(F, a, -1, b, 1, -cf); plane(F, a, 1, b, 1, cf);
      }
    }
  }
  // upwinded advection (lopsidediff.f90:321-481) and KO (kodiss.f90:190-207)
  __device__ __forceinline__ void adv(int F, double v) const {
    const Coef<double>& C = A->C.t;
    const int id[3] = {i, j, k};
    if (G.lop) {
      for (int d = 0; d < 3; ++d) {
        const double b = S.get(F_BETAX + d, i, j, k);
        if (b == 0.0) continue;
        // weights w[o + 3], o = -3 .. 3, of the branch the forward takes
        double w[7] = {0, 0, 0, 0, 0, 0, 0};
        const int idx = id[d], lo = G.lo3[d], hi = G.hi[d];
        bool any = true;
        auto up = [&](double s) { w[2] += -3 * s; w[3] += -10 * s; w[4] += 18 * s; w[5] += -6 * s; w[6] += s; };
        auto cen = [&](double s) { w[1] += s; w[2] += -8 * s; w[4] += 8 * s; w[5] += -s; };
        auto dn = [&](double s) { w[4] += -3 * s; w[3] += -10 * s; w[2] += 18 * s; w[1] += -6 * s; w[0] += s; };
        if (b > 0) {
          if (idx + 3 <= hi) up(1);
          else if (idx + 2 <= hi) cen(1);
          else if (idx + 1 <= hi) dn(-1);
          else any = false;
        } else {
          if (idx - 3 >= lo) dn(-1);
          else if (idx - 2 >= lo) cen(1);
          else if (idx - 1 >= lo) up(1);
          else any = false;
        }
        if (!any) continue;
        const double bd = b * C.d12[d];
        double u = 0.0;
        for (int o = -3; o <= 3; ++o) {
          if (w[o + 3] == 0.0) continue;
          line(F, d, o, v * bd * w[o + 3]);
          u += w[o + 3] * S.get(F, i + (d == 0 ? o : 0), j + (d == 1 ? o : 0), k + (d == 2 ? o : 0));
        }
        S.add(F_BETAX + d, i, j, k, v * C.d12[d] * u);   // the shift as the advecting velocity
      }
    }
    if (G.ko) {
      const double w[7] = {1, -6, 15, -20, 15, -6, 1};
      for (int d = 0; d < 3; ++d) {
        const double c = C.ko / C.h[d] * v;
        for (int o = -3; o <= 3; ++o) line(F, d, o, c * w[o + 3]);
      }
    }
  }

  __device__ __forceinline__ void db(int s, double v) const {
    const int F = slot_field(s), c = s - doff(F), n = dslots(F);
    if (c == n - 1) adv(F, v);
    else if (c < 3) grad(F, c, v);
    else hess(F, c - 3, v);
  }
};

// Writes of the generated VJP: the centre adjoint (added at the point) and the
// D-slot adjoints (stored, then scattered by k_stencil_vjp).
struct VjpStore {
  const AdjBlock* A;
  double* Db;   // D-slot adjoints, same layout as D
  long long p;
  __device__ __forceinline__ void cb(int F, double v) const { atomicAdd(A->Xb + F * A->b.fs + p, v); }
  __device__ __forceinline__ void db(int s, double v) const { Db[s * A->dfs + p] = v; }
};

__device__ __forceinline__ bool on_face_point(const BlockView& b, int i, int j, int k) {
  const int fm = b.face_mask;
  return ((fm & 1) && i == b.ex[0] - 1) || ((fm & 2) && j == b.ex[1] - 1) || ((fm & 4) && k == b.ex[2] - 1) ||
         ((fm & 8) && i == 0) || ((fm & 16) && j == 0) || ((fm & 32) && k == 0);
}

// Pointwise VJP of the right-hand side at the interior (non-face) points:
// centre adjoints into Xb, D-slot adjoints into Db.  Db must start at zero
// (face points leave their slots untouched).
__global__ void __launch_bounds__(128) k_rhs_vjp(const AdjBlock* __restrict__ blocks, double* Db) {
  const AdjBlock& A = blocks[blockIdx.y];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < A.npts;
       p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    point_ijk(p, A.b.ex, i, j, k);
    if (on_face_point(A.b, i, j, k)) continue;
    VjpIn in{&A, p, 0.0};
    VjpStore out{&A, Db, p};
    rhs_vjp_bssn<double>(in, out);
  }
}

// Transpose of the stencil pass: every D-slot adjoint at a point scattered onto
// the field values its stencil read (nslots of the layout: 135 BSSN).
__global__ void __launch_bounds__(128) k_stencil_vjp(const AdjBlock* __restrict__ blocks, const double* Db,
                                                     int nslots) {
  const AdjBlock& A = blocks[blockIdx.y];
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < A.npts;
       p += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    point_ijk(p, A.b.ex, i, j, k);
    if (on_face_point(A.b, i, j, k)) continue;
    VjpOut out{&A, p, i, j, k, point_gates(A.b, i, j, k), Scatter{&A}};
#pragma unroll 1
    for (int s = 0; s < nslots; ++s) {
      const double v = Db[s * A.dfs + p];
      if (v != 0.0) out.db(s, v);
    }
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
// adjoints into Xb, D-slot adjoints into Db (scattered by k_stencil_vjp).
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
struct EnfIn {
  const double* Z;
  const double* Eb;
  long long fs, p;
  __device__ __forceinline__ double c(int m) const { return Z[(F_GXX + m) * fs + p]; }
  __device__ __forceinline__ double d(int) const { return 0.0; }
  __device__ __forceinline__ double rb(int m) const { return Eb[(F_GXX + m) * fs + p]; }
};
struct EnfOut {
  double* Zb;
  long long fs, p;
  __device__ __forceinline__ void cb(int m, double v) { Zb[(F_GXX + m) * fs + p] = v; }
  __device__ __forceinline__ void db(int, double) {}
};

// Zb = mask(Z) * E'(Z)^T Eb (chi masked where the floor held Z at chitiny).
__global__ void __launch_bounds__(128) k_enforce_vjp(const double* __restrict__ Z, const double* __restrict__ Eb,
                                                     double* __restrict__ Zb, long long n, long long fs,
                                                     double chitiny, int enforce) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    for (int f = 0; f < NFIELDS_BSSN; ++f)
      if (!enforce || f < F_GXX || f > F_AZZ) Zb[f * fs + p] = Eb[f * fs + p];
    if (enforce) {
      EnfIn in{Z, Eb, fs, p};
      EnfOut out{Zb, fs, p};
      enforce_vjp<double>(in, out);
    }
    if (Z[F_CHI * fs + p] == chitiny) Zb[F_CHI * fs + p] = 0.0;
  }
}

}  // namespace amss
