// substep_staged.cuh -- the pointwise pass of the split RK4 substep, staged
// through shared memory by bulk asynchronous copies.
//
// The pointwise pass needs, per point, 135 stencil terms (D slots), the 24
// centre values of the stage input, u0 and the RK accumulator K: ~200 words
// read once each.  Issued as ordinary loads from 255-register threads, too few
// of them are in flight to cover HBM latency.  Here one CTA takes a tile of
// STILE consecutive points of a block; lanes of warp 0 issue one
// cp.async.bulk per (array, tile) row -- every row is STILE contiguous words
// of one field or slot, 16-byte aligned because field and slot strides are
// multiples of 64 elements -- completing on one mbarrier.  The whole tile's
// inputs are then in shared memory, and the RHS reads them with no global
// latency.  Several CTAs per SM overlap one tile's copies with another's
// arithmetic.  The mbarrier wait is bounded: on timeout the kernel records
// ST_TIMEOUT, waits (bounded) for its copies to land and returns.
//
// Outer-face points (Sommerfeld / frozen) are left to k_face.
#pragma once
#include <cstdint>

#include "substep_common.cuh"

namespace amss {

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on phase `parity` of `bar`: false after ~2^31 clock cycles.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > (1ll << 31)) return false;
  return true;
}
// One contiguous global -> shared copy completing on `bar` (no multicast).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// Accessor of the staged pointwise pass: centre values and stencil terms from
// the tile in shared memory.  Only centre values exist (v ignores offsets): the
// split RHS reads neighbours through the D slots alone.
template <typename T, typename SI>
struct SPt {
  static constexpr bool kPre = true;
  using elem = SI;
  const SI* cs;         // centre values, [24][STILE]
  const double* side;   // FP64 chi, alpha of an FP32 stage input, [2][STILE]
  const T* ds;          // D slots, [D_SLOTS][STILE]
  int l;                // lane = point in the tile
  long long p;
  int i, j, k;
  template <typename U, int F>
  __device__ __forceinline__ U v(int, int, int) const {
    if constexpr (sizeof(SI) == 4 && wide_field<F>()) return (U)side[side_slot(F) * STILE + l];
    else return (U)cs[F * STILE + l];
  }
  template <typename U>
  __device__ __forceinline__ U dv(int slot) const { return (U)ds[slot * STILE + l]; }
};

// RK4 epilogue reading u0 and K from the staged tile (cf. EpiRK).
template <typename T, typename SO>
struct EpiRKS {
  const double* u0s;   // [24][STILE]
  const double* Ks;    // [24][STILE] (sub >= 1)
  int l;
  double* K;
  SO* out;
  double* out_side;
  long long fs, p;
  int sub;
  bool enforce;
  RKConst c;
  double g[6], a[6];

  template <int F>
  __device__ __forceinline__ void put(T kv) {
    const long long o = F * fs + p;
    const double k = (double)kv;
    const double u = u0s[F * STILE + l];
    double r;
    if (sub == 0) {
      r = u + c.half_dt * k;
      K[o] = k;
    } else if (sub == 1) {
      K[o] = Ks[F * STILE + l] + 2.0 * k;
      r = u + c.half_dt * k;
    } else if (sub == 2) {
      K[o] = Ks[F * STILE + l] + 2.0 * k;
      r = u + c.dt * k;
    } else {
      r = u + c.sixth_dt * (k + Ks[F * STILE + l]);
    }
    if constexpr (F == F_CHI) {
      if (r < c.chitiny) r = c.chitiny;
    }
    if constexpr (F == F_GXX) g[0] = r;
    else if constexpr (F == F_GXY) g[1] = r;
    else if constexpr (F == F_GXZ) g[2] = r;
    else if constexpr (F == F_GYY) g[3] = r;
    else if constexpr (F == F_GYZ) g[4] = r;
    else if constexpr (F == F_GZZ) g[5] = r;
    else if constexpr (F == F_AXX) a[0] = r;
    else if constexpr (F == F_AXY) a[1] = r;
    else if constexpr (F == F_AXZ) a[2] = r;
    else if constexpr (F == F_AYY) a[3] = r;
    else if constexpr (F == F_AYZ) a[4] = r;
    else if constexpr (F == F_AZZ) a[5] = r;
    else if constexpr (sizeof(SO) == 4 && wide_field<F>()) out_side[side_slot(F) * fs + p] = r;
    else out[o] = (SO)r;
  }
  __device__ __forceinline__ void finish() {
    if (enforce) enforce_ga_point(g, a);
    out[F_GXX * fs + p] = (SO)g[0]; out[F_GXY * fs + p] = (SO)g[1]; out[F_GXZ * fs + p] = (SO)g[2];
    out[F_GYY * fs + p] = (SO)g[3]; out[F_GYZ * fs + p] = (SO)g[4]; out[F_GZZ * fs + p] = (SO)g[5];
    out[F_AXX * fs + p] = (SO)a[0]; out[F_AXY * fs + p] = (SO)a[1]; out[F_AXZ * fs + p] = (SO)a[2];
    out[F_AYY * fs + p] = (SO)a[3]; out[F_AYZ * fs + p] = (SO)a[4]; out[F_AZZ * fs + p] = (SO)a[5];
  }
};

// Shared-memory bytes of one staged tile (D slots, stage input + FP64 side,
// u0, K) plus the mbarrier.
template <typename T, typename SI>
__host__ __device__ constexpr size_t staged_smem_bytes() {
  return (size_t)D_SLOTS * STILE * sizeof(T) + (size_t)24 * STILE * sizeof(SI) +
         (sizeof(SI) == 4 ? (size_t)2 * STILE * sizeof(double) : 0) + (size_t)2 * 24 * STILE * sizeof(double) + 16;
}

template <typename T, typename SI, typename SO, bool SYMM>
__global__ void __launch_bounds__(STILE) k_substep_staged(const StepBlock<T>* __restrict__ blocks,
                                                          const int2* __restrict__ tiles, int ntiles, int sub,
                                                          RKConst rk, int enforce, unsigned* status,
                                                          const T* __restrict__ D, long long dfs) {
  extern __shared__ __align__(128) unsigned char stage_smem[];
  T* Ds = reinterpret_cast<T*>(stage_smem);
  SI* Cs = reinterpret_cast<SI*>(stage_smem + (size_t)D_SLOTS * STILE * sizeof(T));
  double* Ss = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(Cs) + (size_t)24 * STILE * sizeof(SI));
  double* Us = Ss + (sizeof(SI) == 4 ? 2 * STILE : 0);
  double* Ks = Us + 24 * STILE;
  uint64_t* bar = reinterpret_cast<uint64_t*>(Ks + 24 * STILE);
  __shared__ int timed_out;

  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    timed_out = 0;
  }
  __syncthreads();
  unsigned parity = 0;
  const int lane = threadIdx.x;
  const bool stage_in = sub != 0;                   // sub 0 reads u0 as its input
  const bool stage_side = stage_in && sizeof(SI) == 4;
  const bool stage_K = sub != 0;

  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 tile = tiles[t];
    const StepBlock<T>& B = blocks[tile.x];
    const long long p0 = tile.y;
    const int cur = B.lvl[0];
    const long long fs = B.b.fs;
    double* u0 = B.tl[cur];
    const SI* in = sub == 0 ? (const SI*)u0 : (const SI*)B.stage[sub == 2 ? 1 : 0];
    const double* in_side = sub == 0 ? nullptr : B.side[sub == 2 ? 1 : 0];

    // ---- stage the tile: warp 0 issues one bulk copy per row ----
    if (threadIdx.x < 32) {
      const int nD = D_SLOTS, nC = stage_in ? 24 : 0, nS = stage_side ? 2 : 0, nU = 24, nK = stage_K ? 24 : 0;
      const int rows = nD + nC + nS + nU + nK;
      if (lane == 0) {
        const unsigned bytes = (unsigned)(nD * STILE * sizeof(T) + nC * STILE * sizeof(SI) +
                                          (nS + nU + nK) * STILE * sizeof(double));
        mbar_arrive_expect_tx(bar, bytes);
      }
      __syncwarp();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      const T* dsrc = D + B.doff + p0;
      for (int r = lane; r < rows; r += 32) {
        int q = r;
        if (q < nD) { bulk_load(Ds + q * STILE, dsrc + q * dfs, STILE * sizeof(T), bar); continue; }
        q -= nD;
        if (q < nC) { bulk_load(Cs + q * STILE, in + q * fs + p0, STILE * sizeof(SI), bar); continue; }
        q -= nC;
        if (q < nS) { bulk_load(Ss + q * STILE, in_side + q * fs + p0, STILE * sizeof(double), bar); continue; }
        q -= nS;
        if (q < nU) { bulk_load(Us + q * STILE, u0 + q * fs + p0, STILE * sizeof(double), bar); continue; }
        q -= nU;
        bulk_load(Ks + q * STILE, B.K + q * fs + p0, STILE * sizeof(double), bar);
      }
    }
    if (threadIdx.x == 0) {
      if (!mbar_wait_bounded(bar, parity)) {
        atomicOr(status, ST_TIMEOUT);
        mbar_wait_bounded(bar, parity);   // let copies in flight land before the CTA leaves
        timed_out = 1;
      }
    }
    __syncthreads();
    if (timed_out) return;
    parity ^= 1u;

    // ---- one point per thread ----
    const long long p = p0 + lane;
    if (p < B.npts) {
      SO* out = sub == 3 ? (SO*)B.tl[(cur + 1) % 3] : (SO*)B.stage[sub == 1 ? 1 : 0];
      double* out_side = sub == 3 ? nullptr : B.side[sub == 1 ? 1 : 0];
      int i, j, k;
      point_ijk(p, B.b.ex, i, j, k);
      const int fm = B.b.face_mask;
      const bool on_face = ((fm & 1) && i == B.b.ex[0] - 1) || ((fm & 2) && j == B.b.ex[1] - 1) ||
                           ((fm & 4) && k == B.b.ex[2] - 1) || ((fm & 8) && i == 0) || ((fm & 16) && j == 0) ||
                           ((fm & 32) && k == 0);
      unsigned st;
      if (!on_face) {
        SPt<T, SI> q;
        q.cs = stage_in ? Cs : reinterpret_cast<const SI*>(Us);   // sub 0: SI is double, the input is u0
        q.side = Ss;
        q.ds = Ds;
        q.l = lane;
        q.p = p;
        q.i = i;
        q.j = j;
        q.k = k;
        EpiRKS<T, SO> epi;
        epi.u0s = Us;
        epi.Ks = Ks;
        epi.l = lane;
        epi.K = B.K;
        epi.out = out;
        epi.out_side = out_side;
        epi.fs = fs;
        epi.p = p;
        epi.sub = sub;
        epi.enforce = enforce != 0;
        epi.c = rk;
        const PointGates G = point_gates(B.b, i, j, k);
        RhsAux aux{};
        st = bssn_rhs_point<T, SI, SYMM, false>(q, B.C, G, aux, epi);
      } else {
        st = 0;   // outer-face points: k_face
      }
      if (st) atomicOr(status, st);
    }
    __syncthreads();   // the tile's shared memory is reused by the next copies
  }
}

}  // namespace amss
