// stencil.cuh -- point access and finite-difference stencils of the BSSN kernels.
//
// One thread owns one grid point (i, j, k) of one block.  Stencil values are
// read straight from HBM/L2 through the read-only path; the stencil formulas
// and their association order are those of diff_new.f90:946-1528
// (fderivs/fdderivs, "for bam comparison" branch), lopsidediff.f90:321-481
// and kodiss.f90:190-207, so that FP64 results agree with the reference to
// round-off.
#pragma once
#include <type_traits>

#include "amss_common.cuh"

namespace amss {

// Per-block stencil coefficients, computed on the host in double exactly as
// the Fortran computes them (e.g. d12dx = ONE/F12/dX) and then cast to T.
template <typename T>
struct Coef {
  T d12[3];          // 1/12/dx
  T d2[3];           // 1/2/dx
  T Fdd[3];          // (1/12)/(dx*dx)
  T Sdd[3];          // 1/(dx*dx)
  T Fxy, Fxz, Fyz;   // (1/144)/(dx*dy)
  T Sxy, Sxz, Syz;   // 0.25/(dx*dy)
  T h[3];            // dx itself (KO divides by it)
  T hinv[3];         // 1/dx, used instead of the division when every dx is a power of two (exact)
  int hpow2;
  T ko;              // eps/64
};

// An FP32 copy of a field f costs ~6e-8 |f| absolute, which a second
// derivative turns into an RHS error of ~6e-8 |f| (4 / dx^2), a stencil's
// cancellation of the field's own size.  chi and alpha carry O(1)
// backgrounds; the shift grows to O(0.1 - 1) near the punctures and its
// second derivatives drive Gamma~^i (gamma~^jk d_j d_k beta^i) and through it
// B^i.  In the mixed form these five fields therefore keep FP64 stage storage
// ("side" arrays, slots chi, alpha, beta^x, beta^y, beta^z) and FP64 stencil
// arithmetic, whose results are rounded only once, relative to the
// derivative itself; every other field is FP32.
template <int F>
__host__ __device__ constexpr bool wide_field() {
  return F == F_CHI || F == F_LAP || F == F_BETAX || F == F_BETAY || F == F_BETAZ;
}
__host__ __device__ constexpr bool is_wide(int F) {
  return F == F_CHI || F == F_LAP || F == F_BETAX || F == F_BETAY || F == F_BETAZ;
}
__host__ __device__ constexpr int side_slot(int F) {
  return F == F_CHI ? 0 : (F == F_LAP ? 1 : 2 + (F - F_BETAX));
}
constexpr int kSideFields = 5;   // FP64 stage fields of the mixed form
static_assert(side_slot(F_BETAX) == 2, "interp.cuh reads the shift from side slot 2");

// Coefficients in the arithmetic type and in FP64 (for the wide fields).
template <typename T>
struct Coefs {
  Coef<T> t;
  Coef<double> d;
};
template <typename A, typename T>
__device__ __forceinline__ const Coef<A>& pick(const Coefs<T>& C) {
  if constexpr (std::is_same_v<A, T>) return C.t;
  else return C.d;
}

// Point accessor.  With SYMM == false, offsets are applied directly: callers
// only step outside [0, ex) where the reference reads its symmetry pad.  With
// SYMM == true every access mirrors negative indices cell-centred,
// f(-m) = f(m-1) * parity (fmisc.f90:877-901), which also covers that pad.
template <typename SI, bool SYMM>
struct Pt {
  static constexpr bool kPre = false;
  using elem = SI;
  const SI* __restrict__ base;  // field 0 of the block
  const double* __restrict__ side;  // FP64 side slots (chi, alpha, beta^i) when SI is float (else unused)
  long long fs;                 // field stride
  long long p;                  // linear index of the point
  long long sy, sz;             // strides of j and k
  int i, j, k;                  // 0-based indices
  int ex0, ex1, ex2;

  template <int F>
  __device__ __forceinline__ auto ld(long long idx) const {
    if constexpr (sizeof(SI) == 4 && wide_field<F>()) return __ldg(side + side_slot(F) * fs + idx);
    else return __ldg(base + F * fs + idx);
  }
  template <typename T, int F>
  __device__ __forceinline__ T v(int di, int dj, int dk) const {
    if constexpr (!SYMM) {
      return (T)ld<F>(p + di + dj * sy + dk * sz);
    } else {
      int ii = i + di, jj = j + dj, kk = k + dk;
      bool neg = false;
      if (ii < 0) { ii = -ii - 1; neg ^= (soa_sign(F, 0) < 0); }
      if (jj < 0) { jj = -jj - 1; neg ^= (soa_sign(F, 1) < 0); }
      if (kk < 0) { kk = -kk - 1; neg ^= (soa_sign(F, 2) < 0); }
      T x = (T)ld<F>(ii + jj * sy + kk * sz);
      return neg ? -x : x;
    }
  }
  // value with the pad rule even when SYMM == false (lopsided reads index -1)
  template <typename T, int F>
  __device__ __forceinline__ T vpad(int di, int dj, int dk) const {
    int ii = i + di, jj = j + dj, kk = k + dk;
    bool neg = false;
    if (ii < 0) { ii = -ii - 1; neg ^= (soa_sign(F, 0) < 0); }
    if (jj < 0) { jj = -jj - 1; neg ^= (soa_sign(F, 1) < 0); }
    if (kk < 0) { kk = -kk - 1; neg ^= (soa_sign(F, 2) < 0); }
    T x = (T)ld<F>(ii + jj * sy + kk * sz);
    return neg ? -x : x;
  }
};

// ---- precomputed stencil terms (split form) ----------------------------------
// The stencil pass (deriv.cuh) stores, per point and field, what the RHS needs
// of that field's neighbourhood: gradient (3), Hessian (6: xx xy xz yy yz zz)
// and "adv" = upwinded advection + eps/64 * KO line sums -- 10 values for the
// shift, chi, the metric and the lapse, 4 for trK and Gamma^i (gradient, adv),
// 1 for A~ij and B^i (adv): 135 slots in all (Z4c: + 4 for Theta).
__host__ __device__ constexpr int dslots(int F) {
  return (F == F_BETAX || F == F_BETAY || F == F_BETAZ || F == F_CHI || F == F_LAP || (F >= F_GXX && F <= F_GZZ))
             ? 10
             : ((F == F_TRK || F == F_GAMX || F == F_GAMY || F == F_GAMZ || F == F_TZ) ? 4 : 1);
}
__host__ __device__ constexpr int doff(int F) {
  int o = 0;
  for (int f = 0; f < F; ++f) o += dslots(f);
  return o;
}
constexpr int D_SLOTS = 135;
static_assert(doff(24) == D_SLOTS, "D slot layout");
// Z4c: Theta's gradient and adv follow (slots 135-138)
constexpr int D_SLOTS_Z4C = D_SLOTS + 4;
static_assert(doff(F_TZ) == D_SLOTS && doff(F_TZ + 1) == D_SLOTS_Z4C, "Z4c D slot layout");

#ifndef AMSS_D_STREAMING   // the D array marked evict-first: bit 0 its stores, bit 1 its loads
#define AMSS_D_STREAMING 3
#endif

// Accessor of the pointwise pass: centre values from the stage input (Pt),
// stencil terms from the D array written by the stencil pass.
template <typename SI, bool SYMM, typename DT>
struct DPt : Pt<SI, SYMM> {
  static constexpr bool kPre = true;
  const DT* __restrict__ d;   // slot 0 of this point's block (add slot * dfs + p)
  long long dfs;              // slot stride
  template <typename T>
  __device__ __forceinline__ T dv(int slot) const {
#if AMSS_D_STREAMING & 2
    return (T)__ldcs(d + slot * dfs + this->p);
#else
    return (T)__ldg(d + slot * dfs + this->p);
#endif
  }
};

template <int D>
__device__ __forceinline__ constexpr int ax(int d) { return D == d ? 1 : 0; }

// ---- first derivatives (fderivs), one direction D ---------------------------
// 4th order: d12 * (f(-2) - 8 f(-1) + 8 f(+1) - f(+2))
template <typename T, int F, int D, typename P>
__device__ __forceinline__ T d1o4(const P& q, const Coef<T>& C) {
  const T EIT = T(8);
  return C.d12[D] * (q.template v<T, F>(-2 * ax<D>(0), -2 * ax<D>(1), -2 * ax<D>(2)) -
                     EIT * q.template v<T, F>(-ax<D>(0), -ax<D>(1), -ax<D>(2)) +
                     EIT * q.template v<T, F>(ax<D>(0), ax<D>(1), ax<D>(2)) -
                     q.template v<T, F>(2 * ax<D>(0), 2 * ax<D>(1), 2 * ax<D>(2)));
}
// 2nd order: d2 * (-f(-1) + f(+1))
template <typename T, int F, int D, typename P>
__device__ __forceinline__ T d1o2(const P& q, const Coef<T>& C) {
  return C.d2[D] * (-q.template v<T, F>(-ax<D>(0), -ax<D>(1), -ax<D>(2)) +
                    q.template v<T, F>(ax<D>(0), ax<D>(1), ax<D>(2)));
}

// Gradient of field F with the reference's joint order gate: ord 2 = 4th order,
// 1 = 2nd order, 0 = derivative is zero (diff_new.f90:1084-1096).
template <typename T, int F, typename P>
__device__ __forceinline__ void grad_a(const P& q, const Coef<T>& C, int ord, T& fx, T& fy, T& fz) {
  if (ord == 2) {
    fx = d1o4<T, F, 0>(q, C); fy = d1o4<T, F, 1>(q, C); fz = d1o4<T, F, 2>(q, C);
  } else if (ord == 1) {
    fx = d1o2<T, F, 0>(q, C); fy = d1o2<T, F, 1>(q, C); fz = d1o2<T, F, 2>(q, C);
  } else {
    fx = T(0); fy = T(0); fz = T(0);
  }
}
template <typename T, int F, typename P>
__device__ __forceinline__ void grad(const P& q, const Coefs<T>& C, int ord, T& fx, T& fy, T& fz) {
  if constexpr (P::kPre) {
    fx = q.template dv<T>(doff(F) + 0); fy = q.template dv<T>(doff(F) + 1); fz = q.template dv<T>(doff(F) + 2);
  } else {
    using A = std::conditional_t<wide_field<F>(), double, T>;
    A ax, ay, az;
    grad_a<A, F>(q, pick<A>(C), ord, ax, ay, az);
    fx = (T)ax; fy = (T)ay; fz = (T)az;
  }
}

// ---- second derivatives (fdderivs) ------------------------------------------
template <typename T, int F, int D, typename P>
__device__ __forceinline__ T d2o4(const P& q, const Coef<T>& C) {
  const T F16 = T(16), F30 = T(30);
  return C.Fdd[D] * (-q.template v<T, F>(-2 * ax<D>(0), -2 * ax<D>(1), -2 * ax<D>(2)) +
                     F16 * q.template v<T, F>(-ax<D>(0), -ax<D>(1), -ax<D>(2)) -
                     F30 * q.template v<T, F>(0, 0, 0) -
                     q.template v<T, F>(2 * ax<D>(0), 2 * ax<D>(1), 2 * ax<D>(2)) +
                     F16 * q.template v<T, F>(ax<D>(0), ax<D>(1), ax<D>(2)));
}
template <typename T, int F, int D, typename P>
__device__ __forceinline__ T d2o2(const P& q, const Coef<T>& C) {
  const T TWO = T(2);
  return C.Sdd[D] * (q.template v<T, F>(-ax<D>(0), -ax<D>(1), -ax<D>(2)) - TWO * q.template v<T, F>(0, 0, 0) +
                     q.template v<T, F>(ax<D>(0), ax<D>(1), ax<D>(2)));
}
// mixed derivative in directions (A, B), A < B: 4th order 16-point cross
// stencil / 144 dA dB, rows taken along A and combined along B.
template <typename T, int F, int A, int B, typename P>
__device__ __forceinline__ T row4(const P& q, int ob) {
  const T F8 = T(8);
  return q.template v<T, F>(-2 * ax<A>(0) + ob * ax<B>(0), -2 * ax<A>(1) + ob * ax<B>(1), -2 * ax<A>(2) + ob * ax<B>(2)) -
         F8 * q.template v<T, F>(-ax<A>(0) + ob * ax<B>(0), -ax<A>(1) + ob * ax<B>(1), -ax<A>(2) + ob * ax<B>(2)) +
         F8 * q.template v<T, F>(ax<A>(0) + ob * ax<B>(0), ax<A>(1) + ob * ax<B>(1), ax<A>(2) + ob * ax<B>(2)) -
         q.template v<T, F>(2 * ax<A>(0) + ob * ax<B>(0), 2 * ax<A>(1) + ob * ax<B>(1), 2 * ax<A>(2) + ob * ax<B>(2));
}
template <typename T, int F, int A, int B, typename P>
__device__ __forceinline__ T dmo4(const P& q, T coef) {
  const T F8 = T(8);
  return coef * (row4<T, F, A, B>(q, -2) - F8 * row4<T, F, A, B>(q, -1) + F8 * row4<T, F, A, B>(q, 1) -
                 row4<T, F, A, B>(q, 2));
}
template <typename T, int F, int A, int B, typename P>
__device__ __forceinline__ T dmo2(const P& q, T coef) {
  return coef * (q.template v<T, F>(-ax<A>(0) - ax<B>(0), -ax<A>(1) - ax<B>(1), -ax<A>(2) - ax<B>(2)) -
                 q.template v<T, F>(ax<A>(0) - ax<B>(0), ax<A>(1) - ax<B>(1), ax<A>(2) - ax<B>(2)) -
                 q.template v<T, F>(-ax<A>(0) + ax<B>(0), -ax<A>(1) + ax<B>(1), -ax<A>(2) + ax<B>(2)) +
                 q.template v<T, F>(ax<A>(0) + ax<B>(0), ax<A>(1) + ax<B>(1), ax<A>(2) + ax<B>(2)));
}

// Hessian of F: fxx fxy fxz fyy fyz fzz (fdderivs output order).
template <typename T, int F, typename P>
__device__ __forceinline__ void hess_a(const P& q, const Coef<T>& C, int ord, T& fxx, T& fxy, T& fxz, T& fyy,
                                       T& fyz, T& fzz) {
  if (ord == 2) {
    fxx = d2o4<T, F, 0>(q, C); fyy = d2o4<T, F, 1>(q, C); fzz = d2o4<T, F, 2>(q, C);
    fxy = dmo4<T, F, 0, 1>(q, C.Fxy); fxz = dmo4<T, F, 0, 2>(q, C.Fxz); fyz = dmo4<T, F, 1, 2>(q, C.Fyz);
  } else if (ord == 1) {
    fxx = d2o2<T, F, 0>(q, C); fyy = d2o2<T, F, 1>(q, C); fzz = d2o2<T, F, 2>(q, C);
    fxy = dmo2<T, F, 0, 1>(q, C.Sxy); fxz = dmo2<T, F, 0, 2>(q, C.Sxz); fyz = dmo2<T, F, 1, 2>(q, C.Syz);
  } else {
    fxx = fxy = fxz = fyy = fyz = fzz = T(0);
  }
}
template <typename T, int F, typename P>
__device__ __forceinline__ void hess(const P& q, const Coefs<T>& C, int ord, T& fxx, T& fxy, T& fxz, T& fyy,
                                     T& fyz, T& fzz) {
  if constexpr (P::kPre) {
    const int o = doff(F) + 3;
    fxx = q.template dv<T>(o); fxy = q.template dv<T>(o + 1); fxz = q.template dv<T>(o + 2);
    fyy = q.template dv<T>(o + 3); fyz = q.template dv<T>(o + 4); fzz = q.template dv<T>(o + 5);
  } else {
    using A = std::conditional_t<wide_field<F>(), double, T>;
    A a[6];
    hess_a<A, F>(q, pick<A>(C), ord, a[0], a[1], a[2], a[3], a[4], a[5]);
    fxx = (T)a[0]; fxy = (T)a[1]; fxz = (T)a[2]; fyy = (T)a[3]; fyz = (T)a[4]; fzz = (T)a[5];
  }
}

// ---- upwinded advection (lopsided), one direction ---------------------------
// Returns r + beta * D^upwind f along D following lopsidediff.f90:321-481;
// `add1` is 1 when the advected array is the full metric g = d + 1.
// lo/hi are the reference's imin/imax in 0-based form.
template <typename T, int F, int D, typename P>
__device__ __forceinline__ T lop_dir(const P& q, const Coefs<T>& CC, T r, T b, int idx, int lo, int hi, T add1) {
  using A = std::conditional_t<wide_field<F>(), double, T>;
  const Coef<A>& C = pick<A>(CC);
  const A F3 = A(3), F10 = A(10), F18 = A(18), F6 = A(6), EIT = A(8);
  auto f = [&](int o) -> A {
    // FP32: the stencil of the offset d, not of d + 1 (the weights sum to zero,
    // and 1 + d in FP32 keeps only ~6e-8 of d)
    if constexpr (sizeof(A) == 4) return q.template vpad<A, F>(o * ax<D>(0), o * ax<D>(1), o * ax<D>(2));
    else return q.template vpad<A, F>(o * ax<D>(0), o * ax<D>(1), o * ax<D>(2)) + A(add1);
  };
  const A bd = A(b) * C.d12[D];
  if constexpr (std::is_same_v<A, T>) {
    if (b > T(0)) {
      if (idx + 3 <= hi)
        r = r + bd * (-F3 * f(-1) - F10 * f(0) + F18 * f(1) - F6 * f(2) + f(3));
      else if (idx + 2 <= hi)
        r = r + bd * (f(-2) - EIT * f(-1) + EIT * f(1) - f(2));
      else if (idx + 1 <= hi)
        r = r - bd * (-F3 * f(1) - F10 * f(0) + F18 * f(-1) - F6 * f(-2) + f(-3));
    } else if (b < T(0)) {
      if (idx - 3 >= lo)
        r = r - bd * (-F3 * f(1) - F10 * f(0) + F18 * f(-1) - F6 * f(-2) + f(-3));
      else if (idx - 2 >= lo)
        r = r + bd * (f(-2) - EIT * f(-1) + EIT * f(1) - f(2));
      else if (idx - 1 >= lo)
        r = r + bd * (-F3 * f(-1) - F10 * f(0) + F18 * f(1) - F6 * f(2) + f(3));
    }
    return r;
  } else {
    A d = A(0);
    if (b > T(0)) {
      if (idx + 3 <= hi) d = bd * (-F3 * f(-1) - F10 * f(0) + F18 * f(1) - F6 * f(2) + f(3));
      else if (idx + 2 <= hi) d = bd * (f(-2) - EIT * f(-1) + EIT * f(1) - f(2));
      else if (idx + 1 <= hi) d = -bd * (-F3 * f(1) - F10 * f(0) + F18 * f(-1) - F6 * f(-2) + f(-3));
    } else if (b < T(0)) {
      if (idx - 3 >= lo) d = -bd * (-F3 * f(1) - F10 * f(0) + F18 * f(-1) - F6 * f(-2) + f(-3));
      else if (idx - 2 >= lo) d = bd * (f(-2) - EIT * f(-1) + EIT * f(1) - f(2));
      else if (idx - 1 >= lo) d = bd * (-F3 * f(-1) - F10 * f(0) + F18 * f(1) - F6 * f(2) + f(3));
    }
    return r + (T)d;
  }
}

// ---- Kreiss-Oliger, combined directions (kodiss.f90:190-207) ----------------
template <typename T, int F, int D, typename P>
__device__ __forceinline__ T ko_line(const P& q) {
  const T SIX = T(6), FIT = T(15), TWT = T(20);
  auto f = [&](int o) -> T { return q.template v<T, F>(o * ax<D>(0), o * ax<D>(1), o * ax<D>(2)); };
  return (f(-3) + f(3)) - SIX * (f(-2) + f(2)) + FIT * (f(-1) + f(1)) - TWT * f(0);
}

// The same line sum in FP64 with every operation rounded as written (no
// contraction into FMA), i.e. as the Fortran evaluates it.  ADD1: sum f + 1,
// where the reference dissipates the full diagonal metric g = d + 1
// (Z4c_rhs.f90:1240-1245).  A KO term acting on O(1e-8)
// noise in an O(1) field is a difference of O(1) values, so any other
// rounding differs from the reference's in relative terms far above 1e-12.
template <typename T, bool ADD1, typename FN>
__device__ __forceinline__ T ko_sum_rn(const FN& f) {
  // FP32: always the sum of d (KO annihilates the constant; 1 + d in FP32 keeps ~6e-8 of d)
  if constexpr (sizeof(T) == 8) {
    auto g = [&](int o) {
      if constexpr (ADD1) return __dadd_rn(f(o), 1.0);
      else return (double)f(o);
    };
    double s = __dadd_rn(g(-3), g(3));
    s = __dsub_rn(s, __dmul_rn(6.0, __dadd_rn(g(-2), g(2))));
    s = __dadd_rn(s, __dmul_rn(15.0, __dadd_rn(g(-1), g(1))));
    return __dsub_rn(s, __dmul_rn(20.0, g(0)));
  } else {
    return (f(-3) + f(3)) - T(6) * (f(-2) + f(2)) + T(15) * (f(-1) + f(1)) - T(20) * f(0);
  }
}

template <typename T>
__device__ __forceinline__ T kodiv(T a, const Coef<T>& c, int d) {
  // the reference divides by dx; for dx = 2^k the product with 2^-k is the same number
  if constexpr (sizeof(T) == 8) return c.hpow2 ? a * c.hinv[d] : a / c.h[d];
  else return a * (T(1) / c.h[d]);
}

}  // namespace amss
