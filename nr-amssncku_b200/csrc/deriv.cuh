// deriv.cuh -- the stencil pass of the split RK4 substep.
//
// One CTA takes one field of one (x, y) tile of a block (W x H points, one
// thread per column, W and H per block) and marches through z, over the whole
// block or over the planes [k0, k1) of one z-slab of it.  The planes k .. k+3 of the
// tile plus a 3-cell halo sit in a 5-slot shared-memory ring, filled as the
// reference's padded copy fh of symmetry_bd (fmisc.f90:877-901): cells at
// negative indices hold the mirrored value times the field's parity, cells
// past the block end are never read by the gated stencils and hold 0.  The
// next plane is fetched into registers while the current one is computed,
// so each plane costs one barrier.  The two-CTA form instead copies planes
// straight into a 6-slot ring with cp.async, two planes ahead, where the
// source needs no type conversion.
//
// z-direction work comes from registers: each thread keeps its column
// f(k-3 .. k+3) and the windows of its x- and y-derivatives Dx f, Dy f at
// planes k-2 .. k+2 (4th order) and k-1 .. k+1 (2nd order), each computed
// once, when its plane enters the window.  The mixed
// derivatives with z are formed as Dz(Dx f) and Dz(Dy f): the reference's
// 16-point (4-point) cross stencils of fdderivs are exactly these tensor
// products of its 1-D stencils, so only the rounding of the coefficient
// product differs.  x- and y-lines and the xy cross stencil read the plane.
//
// Per point the pass stores, for the field's kind (stencil.cuh: dslots):
// gradient, Hessian, and one "adv" value = upwinded advection
// (lopsidediff.f90:321-481) + eps/64 * KO line sums (kodiss.f90:190-207).
// The formulas and gates are those of diff_new.f90:946-1528.
#pragma once
#include "bssn_step.cuh"

namespace amss {

// A tile is W x H columns (W <= DWMAX, W * H <= DTHREADS), chosen per block
// (deriv_tile) so that narrow blocks do not leave lanes idle: W = the block's
// x extent split into pieces of at most 64, H = DTHREADS / W rows.
constexpr int DTHREADS = 256;
// Resident CTAs of DTHREADS threads the stencil pass is compiled for.  Two
// forms: occupancy 0, two CTAs (128 registers), and occupancy 1, four CTAs in
// FP64 / three in FP32 arithmetic (64 / 80 registers; the windows spill a few
// hundred bytes to L1): more warps to cover the plane loads, at the price of
// the spills.  Which is faster depends on the level (the autotuner picks).
constexpr int kDerivMinbLow = 2;
#ifndef AMSS_DERIV_MINB_F64
#define AMSS_DERIV_MINB_F64 4
#endif
#ifndef AMSS_DERIV_MINB_F32
#define AMSS_DERIV_MINB_F32 3
#endif
#ifndef AMSS_DERIV_ASYNC   // 1: the plane ring is filled by cp.async where no type conversion is needed
#define AMSS_DERIV_ASYNC 1
#endif
#ifndef AMSS_DERIV_PREFETCH   // planes beyond the register fetch whose tile rows are prefetched into L2 (0: none)
#define AMSS_DERIV_PREFETCH 4
#endif
constexpr int DWMAX = 64;
constexpr int DPLANE = 704;                 // >= (W + 6) (H + 6) for every admissible W
constexpr int DRING = 5;                    // resident planes: k-1 (being replaced), k .. k+3
constexpr int DRING_ASYNC = 6;              // cp.async ring: k .. k+3, k+4 landing, k+5 issued
constexpr int DPER = (DPLANE + DTHREADS - 1) / DTHREADS;   // plane cells per thread

// Tile shape of the stencil pass for a block of x extent ex0.
__host__ __device__ constexpr int deriv_tile_w(int ex0) {
  return (ex0 + (ex0 + DWMAX - 1) / DWMAX - 1) / ((ex0 + DWMAX - 1) / DWMAX);
}
__host__ __device__ constexpr int deriv_tile_h(int ex0) { return DTHREADS / deriv_tile_w(ex0); }
constexpr int kDerivMinEx = 8;              // the split form needs blocks at least this wide in x
constexpr bool deriv_planes_fit(int w) {
  return w > DWMAX || ((w + 6) * (DTHREADS / w + 6) <= DPLANE && deriv_planes_fit(w + 1));
}
static_assert(deriv_planes_fit(kDerivMinEx), "plane buffer too small for a tile shape");

// substep tile of the split form's pointwise pass
constexpr int kPointwiseTile = 128;
// fewest planes of a z-slab of the stencil pass (each slab pays a 7-plane prologue)
constexpr int kMinSlab = 8;

struct DerivItem {
  int block;   // index into the level's StepBlock table
  int x0, y0;  // tile origin (array indices)
  int field;
  int k0 = 0, k1 = 0;   // planes [k0, k1) of the march; k1 == 0: the whole block
  int x1 = 0, y1 = 0;   // columns x < x1, y < y1 only; 0: up to the block's extent
  int w = 0;            // tile width; 0: the block's (StepBlock::dw)
};

// kind of a field's stencil record: 0 gradient + Hessian + adv, 1 gradient + adv, 2 adv
__host__ __device__ constexpr int dkind(int F) { return dslots(F) == 10 ? 0 : (dslots(F) == 4 ? 1 : 2); }

__device__ __forceinline__ int ring_slot(int m) { return (m + 3) % DRING; }   // m >= -3

// Asynchronous copies global -> shared of one 8- or 4-byte cell (zero-filled
// when !valid; the source address is then not read).
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// A stencil term into D: written once here and read once by the pointwise
// pass, so with AMSS_D_STREAMING bit 0 the store is marked evict-first
// (st.global.cs) and leaves L2 to the fields the stencil pass re-reads.
template <typename T>
__device__ __forceinline__ void dstore(T* a, T v) {
#if AMSS_D_STREAMING & 1
  __stcs(a, v);
#else
  *a = v;
#endif
}

// The plane cells one thread fills, with their in-plane offsets and the x/y
// mirror signs, fixed for the whole march.
template <typename A, typename S>
struct PlaneFetch {
  const S* src;
  long long sz;
  int ex2;
  int off[DPER];     // i + j * ex0 of the (mirrored) cell, -1: none / past the end
  unsigned neg;      // bit e: x/y mirroring flips the sign of cell e
  bool zodd;         // field parity in z is odd
  A v[DPER];

  __device__ __forceinline__ void init(const S* s, int F, const int* ex, int x0, int y0, int sx, int np) {
    src = s;
    sz = (long long)ex[0] * ex[1];
    ex2 = ex[2];
    zodd = soa_sign(F, 2) < 0;
    neg = 0;
#pragma unroll
    for (int e = 0; e < DPER; ++e) {
      const int t = threadIdx.x + e * DTHREADS;
      int o = -1;
      if (t < np) {
        int i = x0 - 3 + t % sx, j = y0 - 3 + t / sx;
        bool n = false;
        if (i < 0) { i = -i - 1; n ^= soa_sign(F, 0) < 0; }
        if (j < 0) { j = -j - 1; n ^= soa_sign(F, 1) < 0; }
        if (i < ex[0] && j < ex[1]) o = i + j * ex[0];
        if (n) neg |= 1u << e;
      }
      off[e] = o;
    }
  }
  // issue the loads of plane kk (negative: mirrored, past the end: 0) into w
  __device__ __forceinline__ void fetch_to(int kk, A* w) const {
    int k = kk;
    bool nz = false;
    if (k < 0) { k = -k - 1; nz = zodd; }
    const bool kin = k < ex2;
#pragma unroll
    for (int e = 0; e < DPER; ++e) {
      A x = A(0);
      if (kin && off[e] >= 0) {
        x = (A)__ldg(src + off[e] + k * sz);
        if ((((neg >> e) & 1u) != 0) != nz) x = -x;
      }
      w[e] = x;
    }
  }
  __device__ __forceinline__ void fetch(int kk) { fetch_to(kk, v); }
  __device__ __forceinline__ void store_from(A* slot, int np, const A* w) const {
#pragma unroll
    for (int e = 0; e < DPER; ++e) {
      const int t = threadIdx.x + e * DTHREADS;
      if (t < np) slot[t] = w[e];
    }
  }
  __device__ __forceinline__ void store(A* slot, int np) const { store_from(slot, np, v); }
};

// The same plane cells copied straight into the ring by cp.async when the
// source type is the arithmetic type: no registers hold the plane in flight.
// Cells past the block end are zero-filled by the copy; a mirrored cell is
// negated after its copy lands, by the thread that issued it.
template <typename A>
struct PlaneAsync {
  const A* src;
  long long sz;
  int ex2, np;
  int off[DPER];     // i + j * ex0 of the (mirrored) cell, -1: none / past the end
  unsigned neg;      // bit e: x/y mirroring flips the sign of cell e
  bool zodd;         // field parity in z is odd

  __device__ __forceinline__ void init(const A* s, int F, const int* ex, int x0, int y0, int sx, int n) {
    src = s;
    sz = (long long)ex[0] * ex[1];
    ex2 = ex[2];
    np = n;
    zodd = soa_sign(F, 2) < 0;
    neg = 0;
#pragma unroll
    for (int e = 0; e < DPER; ++e) {
      const int t = threadIdx.x + e * DTHREADS;
      int o = -1;
      if (t < n) {
        int i = x0 - 3 + t % sx, j = y0 - 3 + t / sx;
        bool m = false;
        if (i < 0) { i = -i - 1; m ^= soa_sign(F, 0) < 0; }
        if (j < 0) { j = -j - 1; m ^= soa_sign(F, 1) < 0; }
        if (i < ex[0] && j < ex[1]) o = i + j * ex[0];
        if (m) neg |= 1u << e;
      }
      off[e] = o;
    }
  }
  // issue the copies of plane kk (negative: mirrored, past the end: 0) into slot
  __device__ __forceinline__ void issue(int kk, A* slot) const {
    const int k = kk < 0 ? -kk - 1 : kk;
    const bool kin = k < ex2;
#pragma unroll
    for (int e = 0; e < DPER; ++e) {
      const int t = threadIdx.x + e * DTHREADS;
      if (t < np) {
        const bool ok = kin && off[e] >= 0;
        const A* g = ok ? src + off[e] + k * sz : src;
        if constexpr (sizeof(A) == 8) cp_async8(slot + t, g, ok);
        else cp_async4(slot + t, g, ok);
      }
    }
  }
  // after the copies of plane kk landed: the signs of its mirrored cells
  __device__ __forceinline__ void fix(int kk, A* slot) const {
    const bool nz = kk < 0 && zodd;
    if (!neg && !nz) return;
    const int k = kk < 0 ? -kk - 1 : kk;
    if (k >= ex2) return;
#pragma unroll
    for (int e = 0; e < DPER; ++e) {
      const int t = threadIdx.x + e * DTHREADS;
      if (t < np && off[e] >= 0 && (((neg >> e) & 1u) != 0) != nz) slot[t] = -slot[t];
    }
  }
};

// Upwinded term of one direction (lopsidediff.f90:321-481) over a line f(o),
// o = -3 .. 3 relative to the point; f already includes the +1 of the
// diagonal metric.  bd = beta * d12.
template <typename A, typename FN>
__device__ __forceinline__ A lop_term(const FN& f, A b, A bd, int idx, int lo, int hi) {
  const A F3 = A(3), F10 = A(10), F18 = A(18), F6 = A(6), EIT = A(8);
  if (idx - 3 >= lo && idx + 3 <= hi) {
    // both full-width branches fit: the same arithmetic on the mirrored line,
    // chosen by selects instead of divergent branches
    const bool pos = b > A(0);
    const A fa = pos ? f(-1) : f(1), fb = f(0), fc = pos ? f(1) : f(-1);
    const A fd = pos ? f(2) : f(-2), fe = pos ? f(3) : f(-3);
    const A s = -F3 * fa - F10 * fb + F18 * fc - F6 * fd + fe;
    return pos ? bd * s : (b < A(0) ? -bd * s : A(0));
  }
  A d = A(0);
  if (b > A(0)) {
    if (idx + 3 <= hi) d = bd * (-F3 * f(-1) - F10 * f(0) + F18 * f(1) - F6 * f(2) + f(3));
    else if (idx + 2 <= hi) d = bd * (f(-2) - EIT * f(-1) + EIT * f(1) - f(2));
    else if (idx + 1 <= hi) d = -bd * (-F3 * f(1) - F10 * f(0) + F18 * f(-1) - F6 * f(-2) + f(-3));
  } else if (b < A(0)) {
    if (idx - 3 >= lo) d = -bd * (-F3 * f(1) - F10 * f(0) + F18 * f(-1) - F6 * f(-2) + f(-3));
    else if (idx - 2 >= lo) d = bd * (f(-2) - EIT * f(-1) + EIT * f(1) - f(2));
    else if (idx - 1 >= lo) d = bd * (-F3 * f(-1) - F10 * f(0) + F18 * f(1) - F6 * f(2) + f(3));
  }
  return d;
}

// March one field of one tile.  A: stencil arithmetic type, S: type of the
// field's source array, SI: type of the stage input (for the shift), T: type
// of the D array.
template <typename A, int KIND, bool ASYNC, typename T, typename S, typename SI>
__device__ __forceinline__ void deriv_column(const StepBlock<T>& B, const S* src, const SI* in, const double* bsh,
                                             int F, const DerivItem& it, T* D, long long dfs, A* ring) {
  const Coef<A>& C = pick<A>(B.C);
  const int ex0 = B.b.ex[0], ex1 = B.b.ex[1], ex2 = B.b.ex[2];
  const int x0 = it.x0, y0 = it.y0, k0 = it.k0;
  const int kend = it.k1 > 0 ? it.k1 : ex2;
  const int xend = it.x1 > 0 ? it.x1 : ex0, yend = it.y1 > 0 ? it.y1 : ex1;
  const long long fs = B.b.fs;
  const int W = it.w > 0 ? it.w : B.dw, H = DTHREADS / W;
  const int DSX = W + 6;                     // row stride of the plane buffer
  const int np = DSX * (H + 6);              // cells of one plane (<= DPLANE)
  const int li = threadIdx.x % W, lj = threadIdx.x / W;
  const int i = x0 + li, j = y0 + lj;
  const bool mine = lj < H && i < xend && j < yend;
  const int fm = B.b.face_mask;
  const bool face_xy = ((fm & 1) && i == ex0 - 1) || ((fm & 2) && j == ex1 - 1) || ((fm & 8) && i == 0) ||
                       ((fm & 16) && j == 0);
  // the diagonal metric is advected as g = d + 1 (bssn_rhs.f90:948-953) in FP64,
  // bit-faithful to the reference; FP32 advects d (the constant drops out)
  const A add1 = (sizeof(A) == 8 && (F == F_GXX || F == F_GYY || F == F_GZZ)) ? A(1) : A(0);
  const int o = doff(F);
  T* d = D + B.doff;
  const int own = (lj < H ? lj + 3 : 3) * DSX + (li + 3);   // idle threads read a valid cell

  // ASYNC: cp.async fills the ring where the source needs no conversion (six
  // slots: planes k .. k+3 read, k+4 landing, k+5 issued); otherwise the
  // planes pass through registers (five slots)
  constexpr bool kAsync = ASYNC && sizeof(A) == sizeof(S);
  constexpr int R = kAsync ? DRING_ASYNC : DRING;
  auto rs = [](int m) { return (m + 3) % R; };   // ring slot of plane m >= -3
  PlaneFetch<A, S> P;
  PlaneAsync<A> PA;
  if constexpr (kAsync) PA.init(reinterpret_cast<const A*>(src), F, B.b.ex, x0, y0, DSX, np);
  else P.init(src, F, B.b.ex, x0, y0, DSX, np);

  A c[7];                  // column f(k-3 .. k+3)
  A fx4[5], fy4[5];        // 4th-order Dx f, Dy f at planes k-2 .. k+2 (KIND 0)
  A fx2[3], fy2[3];        // 2nd-order Dx f, Dy f at planes k-1 .. k+1 (KIND 0)

  auto dx4 = [&](const A* q) { return C.d12[0] * (q[-2] - A(8) * q[-1] + A(8) * q[1] - q[2]); };
  auto dy4 = [&](const A* q) { return C.d12[1] * (q[-2 * DSX] - A(8) * q[-DSX] + A(8) * q[DSX] - q[2 * DSX]); };
  auto dx2 = [&](const A* q) { return C.d2[0] * (-q[-1] + q[1]); };
  auto dy2 = [&](const A* q) { return C.d2[1] * (-q[-DSX] + q[DSX]); };

  // prologue: the column gets planes k0-3 .. k0+3 and the derivative windows
  // planes k0-2 .. k0+1.  Register form: the loads of the seven planes are
  // issued together, then the planes enter the ring one at a time.  cp.async
  // form: planes k0-3 .. k0+2 fill the six slots at once; once they are read,
  // k0+3 and k0+4 take the slots of k0-3 and k0-2.
  A pro[kAsync ? 1 : 7][DPER];
  if constexpr (kAsync) {
#pragma unroll
    for (int m = -3; m <= 2; ++m) PA.issue(k0 + m, ring + rs(k0 + m) * DPLANE);
    cp_async_commit();
    cp_async_wait<0>();
#pragma unroll
    for (int m = -3; m <= 2; ++m) PA.fix(k0 + m, ring + rs(k0 + m) * DPLANE);
    __syncthreads();
  } else {
#pragma unroll
    for (int m = -3; m <= 3; ++m) P.fetch_to(k0 + m, pro[m + 3]);
  }
#pragma unroll
  for (int m = -3; m <= 3; ++m) {
    A* slot = ring + rs(k0 + m) * DPLANE;
    if constexpr (kAsync) {
      if (m == 3) {
        __syncthreads();   // planes k0-3, k0-2 are read: their slots take k0+3, k0+4
        PA.issue(k0 + 3, slot);
        cp_async_commit();
        PA.issue(k0 + 4, ring + rs(k0 + 4) * DPLANE);
        cp_async_commit();
        cp_async_wait<1>();
        PA.fix(k0 + 3, slot);
        __syncthreads();
      }
    } else {
      P.store_from(slot, np, pro[m + 3]);
      __syncthreads();
    }
    const A* q = slot + own;
    const A cm = q[0];
#pragma unroll
    for (int t = 0; t < 7; ++t)
      if (t == m + 3) c[t] = cm;
    if constexpr (KIND == 0) {
      if (m >= -2 && m <= 1) {
        const A a4 = dx4(q), b4 = dy4(q), a2 = dx2(q), b2 = dy2(q);
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if (t == m + 2) { fx4[t] = a4; fy4[t] = b4; }
#pragma unroll
        for (int t = 0; t < 2; ++t)
          if (t == m + 1) { fx2[t] = a2; fy2[t] = b2; }
      }
    }
  }

#pragma unroll 1
  for (int k = k0; k < kend; ++k) {
    // in flight while plane k is computed: plane k+4 (registers) or k+5 (cp.async)
    if constexpr (kAsync) {
      PA.issue(k + 5, ring + rs(k + 5) * DPLANE);
      cp_async_commit();
    } else {
      P.fetch(k + 4);
    }
#if AMSS_DERIV_PREFETCH
    {
      // warp 0 asks L2 for the tile rows (with halo) of plane k+4+AMSS_DERIV_PREFETCH,
      // one 128-byte line per lane, so the register fetch of that plane meets L2
      const int kk = k + 4 + AMSS_DERIV_PREFETCH;
      if (threadIdx.x < 32 && kk < ex2 && kk < kend + 3) {
        const int xl = x0 - 3 < 0 ? 0 : x0 - 3, xh = x0 + W + 3 > ex0 ? ex0 : x0 + W + 3;
        const int yl = y0 - 3 < 0 ? 0 : y0 - 3, yh = y0 + H + 3 > ex1 ? ex1 : y0 + H + 3;
        const int lpr = (int)(((xh - xl) * sizeof(S) + 127) / 128);   // lines per row
        for (int t = threadIdx.x; t < lpr * (yh - yl); t += 32) {
          const int r = t / lpr, c = t - r * lpr;
          const char* row = (const char*)(src + xl + (long long)(yl + r) * ex0 + (long long)kk * ex0 * ex1);
          const long long off = (long long)c * 128 < (long long)((xh - xl - 1) * sizeof(S)) ? (long long)c * 128
                                                                                           : (long long)((xh - xl - 1) * sizeof(S));
          asm volatile("prefetch.global.L2 [%0];" ::"l"(row + off));
        }
      }
    }
#endif
    const A* qk = ring + rs(k) * DPLANE + own;
    c[6] = ring[rs(k + 3) * DPLANE + own];
    if constexpr (KIND == 0) {
      const A* q2 = ring + rs(k + 2) * DPLANE + own;
      const A* q1 = ring + rs(k + 1) * DPLANE + own;
      fx4[4] = dx4(q2); fy4[4] = dy4(q2); fx2[2] = dx2(q1); fy2[2] = dy2(q1);
    }
    const bool on_face = face_xy || ((fm & 4) && k == ex2 - 1) || ((fm & 32) && k == 0);
    if (mine && !on_face) {
      const PointGates G = point_gates(B.b, i, j, k);
      const long long p = i + (long long)j * ex0 + (long long)k * ex0 * ex1;
      auto X = [&](int dd) { return qk[dd]; };
      auto Y = [&](int dd) { return qk[dd * DSX]; };
      auto Z = [&](int dd) { return c[3 + dd]; };
      if constexpr (KIND <= 1) {
        A gx = A(0), gy = A(0), gz = A(0);
        if (G.ord == 2) {
          if constexpr (KIND == 0) { gx = fx4[2]; gy = fy4[2]; }
          else { gx = dx4(qk); gy = dy4(qk); }
          gz = C.d12[2] * (Z(-2) - A(8) * Z(-1) + A(8) * Z(1) - Z(2));
        } else if (G.ord == 1) {
          if constexpr (KIND == 0) { gx = fx2[1]; gy = fy2[1]; }
          else { gx = dx2(qk); gy = dy2(qk); }
          gz = C.d2[2] * (-Z(-1) + Z(1));
        }
        dstore(d + (o + 0) * dfs + p, (T)gx);
        dstore(d + (o + 1) * dfs + p, (T)gy);
        dstore(d + (o + 2) * dfs + p, (T)gz);
      }
      if constexpr (KIND == 0) {
        A hxx = A(0), hxy = A(0), hxz = A(0), hyy = A(0), hyz = A(0), hzz = A(0);
        const A F16 = A(16), F30 = A(30), F8 = A(8), TWO = A(2);
        if (G.ord == 2) {
          hxx = C.Fdd[0] * (-X(-2) + F16 * X(-1) - F30 * X(0) - X(2) + F16 * X(1));
          hyy = C.Fdd[1] * (-Y(-2) + F16 * Y(-1) - F30 * Y(0) - Y(2) + F16 * Y(1));
          hzz = C.Fdd[2] * (-Z(-2) + F16 * Z(-1) - F30 * Z(0) - Z(2) + F16 * Z(1));
          auto row = [&](int ob) {
            const A* r = qk + ob * DSX;
            return r[-2] - F8 * r[-1] + F8 * r[1] - r[2];
          };
          hxy = C.Fxy * (row(-2) - F8 * row(-1) + F8 * row(1) - row(2));
          hxz = C.d12[2] * (fx4[0] - F8 * fx4[1] + F8 * fx4[3] - fx4[4]);
          hyz = C.d12[2] * (fy4[0] - F8 * fy4[1] + F8 * fy4[3] - fy4[4]);
        } else if (G.ord == 1) {
          hxx = C.Sdd[0] * (X(-1) - TWO * X(0) + X(1));
          hyy = C.Sdd[1] * (Y(-1) - TWO * Y(0) + Y(1));
          hzz = C.Sdd[2] * (Z(-1) - TWO * Z(0) + Z(1));
          hxy = C.Sxy * (qk[-1 - DSX] - qk[1 - DSX] - qk[-1 + DSX] + qk[1 + DSX]);
          hxz = C.d2[2] * (-fx2[0] + fx2[2]);
          hyz = C.d2[2] * (-fy2[0] + fy2[2]);
        }
        dstore(d + (o + 3) * dfs + p, (T)hxx);
        dstore(d + (o + 4) * dfs + p, (T)hxy);
        dstore(d + (o + 5) * dfs + p, (T)hxz);
        dstore(d + (o + 6) * dfs + p, (T)hyy);
        dstore(d + (o + 7) * dfs + p, (T)hyz);
        dstore(d + (o + 8) * dfs + p, (T)hzz);
      }
      A adv = A(0);
      if (G.lop) {
        // the shift at the point, from the stage input (bsh: its FP64 side
        // slots in the mixed form), rounded to the storage type T of the
        // other fields as the pointwise pass sees it
        const T bx = bsh ? (T)__ldg(bsh + p) : (T)__ldg(in + F_BETAX * fs + p);
        const T by = bsh ? (T)__ldg(bsh + fs + p) : (T)__ldg(in + F_BETAY * fs + p);
        const T bz = bsh ? (T)__ldg(bsh + 2 * fs + p) : (T)__ldg(in + F_BETAZ * fs + p);
        auto Xp = [&](int dd) { return X(dd) + add1; };
        auto Yp = [&](int dd) { return Y(dd) + add1; };
        auto Zp = [&](int dd) { return Z(dd) + add1; };
        adv = lop_term<A>(Xp, (A)bx, (A)bx * C.d12[0], i, G.lo3[0], G.hi[0]);
        adv = adv + lop_term<A>(Yp, (A)by, (A)by * C.d12[1], j, G.lo3[1], G.hi[1]);
        adv = adv + lop_term<A>(Zp, (A)bz, (A)bz * C.d12[2], k, G.lo3[2], G.hi[2]);
      }
      if (G.ko) {
        // Z4c dissipates the full diagonal metric d + 1 (Z4c_rhs.f90:1240-1245)
        const bool ko1 = B.nf == NFIELDS_Z4C && (F == F_GXX || F == F_GYY || F == F_GZZ);
        A ks;
        if (ko1)
          ks = kodiv(ko_sum_rn<A, true>(X), C, 0) + kodiv(ko_sum_rn<A, true>(Y), C, 1) +
               kodiv(ko_sum_rn<A, true>(Z), C, 2);
        else
          ks = kodiv(ko_sum_rn<A, false>(X), C, 0) + kodiv(ko_sum_rn<A, false>(Y), C, 1) +
               kodiv(ko_sum_rn<A, false>(Z), C, 2);
        adv = adv + C.ko * ks;
      }
      dstore(d + (o + dslots(F) - 1) * dfs + p, (T)adv);
    }
    // slide the register windows
#pragma unroll
    for (int t = 0; t < 6; ++t) c[t] = c[t + 1];
    if constexpr (KIND == 0) {
#pragma unroll
      for (int t = 0; t < 4; ++t) { fx4[t] = fx4[t + 1]; fy4[t] = fy4[t + 1]; }
#pragma unroll
      for (int t = 0; t < 2; ++t) { fx2[t] = fx2[t + 1]; fy2[t] = fy2[t + 1]; }
    }
    // plane k+4 is complete for the next iteration: it replaced plane k-1
    // (register form) or landed (cp.async form), and no thread reads that slot
    // in this iteration
    if constexpr (kAsync) {
      cp_async_wait<1>();
      PA.fix(k + 4, ring + rs(k + 4) * DPLANE);
    } else {
      P.store(ring + ring_slot(k + 4) * DPLANE, np);
    }
    __syncthreads();
  }
  // the copies still in flight land before the ring is reused
  if constexpr (kAsync) cp_async_wait<0>();
}

// Stencil pass over a work list of (block, tile, field) items, ordered by
// field so that resident CTAs share one code path.
template <typename T, typename SI, int MINB>
__global__ void __launch_bounds__(DTHREADS, MINB) k_deriv(const StepBlock<T>* __restrict__ blocks,
                                                      const DerivItem* __restrict__ items, int nitems, int sub,
                                                      T* __restrict__ D, long long dfs) {
  extern __shared__ __align__(16) unsigned char smem[];
  // the two-CTA form fills its ring by cp.async; the forms with more CTAs keep
  // the register path, whose smaller ring leaves L1 to their spills
  constexpr bool kAsyncForm = AMSS_DERIV_ASYNC && MINB == kDerivMinbLow;
  for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
    const DerivItem it = items[w];
    const StepBlock<T>& B = blocks[it.block];
    const int cur = B.lvl[0];
    const SI* in = sub == 0 ? (const SI*)B.tl[cur] : (const SI*)B.stage[sub == 2 ? 1 : 0];
    const int F = it.field;
    const long long fs = B.b.fs;
    // the mixed form's stages keep the shift in their FP64 side slots
    const double* bsh = sizeof(SI) == 4 ? B.side[sub == 2 ? 1 : 0] + side_slot(F_BETAX) * fs : nullptr;
    if constexpr (sizeof(T) == 4) {
      if (is_wide(F)) {
        // wide fields of the mixed form: FP64 source (state, or the FP64 side stage) and arithmetic
        const double* src = sizeof(SI) == 4 ? B.side[sub == 2 ? 1 : 0] + side_slot(F) * fs
                                            : (const double*)in + F * fs;
        deriv_column<double, 0, kAsyncForm>(B, src, in, bsh, F, it, D, dfs, reinterpret_cast<double*>(smem));
        __syncthreads();
        continue;
      }
    }
    const SI* src = in + F * fs;
    switch (dkind(F)) {
      case 0: deriv_column<T, 0, kAsyncForm>(B, src, in, bsh, F, it, D, dfs, reinterpret_cast<T*>(smem)); break;
      case 1: deriv_column<T, 1, kAsyncForm>(B, src, in, bsh, F, it, D, dfs, reinterpret_cast<T*>(smem)); break;
      default: deriv_column<T, 2, kAsyncForm>(B, src, in, bsh, F, it, D, dfs, reinterpret_cast<T*>(smem)); break;
    }
    __syncthreads();
  }
}

// Shared memory of k_deriv: the plane ring in the widest arithmetic type, for
// the two-CTA form (cp.async ring) and the others (register path).
constexpr size_t kDerivSmemLow = (size_t)(AMSS_DERIV_ASYNC ? DRING_ASYNC : DRING) * DPLANE * sizeof(double);
constexpr size_t kDerivSmem = (size_t)DRING * DPLANE * sizeof(double);

}  // namespace amss
