// adjoint.cu -- gradient of the Hamiltonian-constraint loss of a BSSN
// evolution with respect to its initial state (amss_adjoint_*).
//
// One level-0 block (the whole patch, Sommerfeld faces), FP64, split form.
// The forward runs the engine's own kernels (stencil pass, pointwise pass,
// face pass) step by step, with enforce_ga applied by a separate pass so the
// pre-enforce stage values Z_s stay available; it keeps a checkpoint of the
// state every `ck` steps.  Loss L = sum over the interior cells (3 cells in
// from every face) of H^2 dV, H the BSSN Hamiltonian constraint.
//
// Backward: per checkpoint segment, from the last, the segment is recomputed
// storing every step's U0 (raw), Z_0..Z_2 and U_new; then each step is
// reversed.  With R_s = F(X_s), X_0 = E(U0), X_{s+1} = E(Z_s),
// Z_s = floor(U0 + c_s R_s) and U_new = floor(U0 + dt/6 (R0 + 2R1 + 2R2 + R3)):
//   Yb = mask(U_new) Ub;  U0b = Yb;  R3b = dt/6 Yb;  R0b = dt/6 Yb;  R1b = R2b = dt/3 Yb
//   s = 3, 2, 1:  Xb_s = F'(X_s)^T R_sb;  Zb = mask(Z_{s-1}) E'(Z_{s-1})^T Xb_s;
//                 U0b += Zb;  R_{s-1}b += c_{s-1} Zb        (c = dt/2, dt/2, dt)
//   U0b += F'(X_0)^T R0b;  Ub(previous step) = E'(U0 raw)^T U0b.
// F'^T is k_rhs_vjp (pointwise, generated) + k_stencil_gather_tiled (stencil
// transpose) + k_face_vjp (Sommerfeld transpose); E'^T and the floor mask are
// k_enforce_vjp.
#include <cmath>
#include <cstdio>
#include <vector>

#include "adjoint.cuh"
#include "amss_b200.h"
#include "dev_util.cuh"

namespace amss {

template <typename T>
Coef<T> make_coef(const double dx[3], double eps);
void block_faces(const int ex[3], const double* X, const double* Y, const double* Z, const double bbox[6],
                 int symmetry, int* face_mask, int* lowsym_mask);
template <typename T, typename SS, bool SYMM, bool SPLIT, bool Z4C>
cudaError_t launch_substep(const void* blocks, const int2* tiles, int ntiles, int sub, RKConst rk, int enforce,
                           unsigned* status, int grid, cudaStream_t s, const void* D, long long dfs);
template <typename T, typename SS, bool SYMM>
cudaError_t launch_face(const void* blocks, const int2* faces, int nfaces, int sub, RKConst rk, int enforce,
                        unsigned* status, cudaStream_t s);
template <typename T, typename SS>
cudaError_t launch_deriv(const void* blocks, const DerivItem* items, int nitems, int sub, void* D, long long dfs,
                         int grid, cudaStream_t s, int occ);

// out = E(in) on the metric / A~ fields; other fields copied.
__global__ void k_enforce_copy(const double* __restrict__ in, double* __restrict__ out, long long n, long long fs) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    double g[6], a[6];
    for (int m = 0; m < 6; ++m) { g[m] = in[(F_GXX + m) * fs + p]; a[m] = in[(F_AXX + m) * fs + p]; }
    enforce_ga_point(g, a);
    for (int f = 0; f < NFIELDS_BSSN; ++f) {
      double v;
      if (f >= F_GXX && f < F_GXX + 6) v = g[f - F_GXX];
      else if (f >= F_AXX && f < F_AXX + 6) v = a[f - F_AXX];
      else v = in[f * fs + p];
      out[f * fs + p] = v;
    }
  }
}

}  // namespace amss

using namespace amss;

struct amss_adjoint {
  int ex[3];
  long long npts = 0, fs = 0;
  double eps = 0.1, chitiny = 1e-5 - 1.0, dx[3] = {0, 0, 0};
  cudaStream_t stream = nullptr;
  unsigned* dstatus = nullptr;
  int* dlvl = nullptr;
  double* dcoord = nullptr;
  StepBlock<double> host_tab[4]{};
  StepBlock<double>* dtab = nullptr;     // 4 tables, one per substep
  AdjBlock host_adj{};
  AdjBlock* dadj = nullptr;
  DerivItem* ditems = nullptr;
  int nitems = 0;
  int2* dtiles = nullptr;
  int ntiles = 0;
  int2* dfaces = nullptr;
  int nfaces = 0;
  double* D = nullptr;                   // stencil terms (D_SLOTS x fs)
  double* Db = nullptr;                  // their adjoints
  double* U = nullptr;                   // state (input of set_state / result of forward)
  double* U0 = nullptr;                  // enforced step start
  double* X[3] = {nullptr, nullptr, nullptr};  // X_1..X_3
  double* K = nullptr;
  double* Zs = nullptr;                  // scratch Z_0..Z_2 for unstored steps (3 states)
  double* H = nullptr;
  double* dloss = nullptr;
  std::vector<double*> ckpt;             // checkpoints
  double* seg = nullptr;                 // segment storage: per step U0raw, Z0, Z1, Z2, Unew
  int seg_cap = 0;
  double* Dseg = nullptr;                // the segment's stencil terms, per step and substep (if HBM allows)
  int dseg_cap = 0;
  bool last_seg_ready = false;           // the forward left the last segment's states (and terms) in seg / Dseg
  double* Ub = nullptr;
  double* U0b = nullptr;
  double* Rb[4] = {nullptr, nullptr, nullptr, nullptr};
  double* Xb = nullptr;
  double dt = 0;
  int nsteps = 0, ck = 1;
  bool forward_done = false;
  long long launches = 0;
};

namespace {

size_t state_bytes(const amss_adjoint* a) { return (size_t)NFIELDS_BSSN * a->fs * sizeof(double); }

int grid_of(long long n) {
  const long long b = (n + 127) / 128;
  return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

// The four substep tables: inputs U0, X1, X2, X3 (enforced), outputs Z0, Z1,
// Z2 (pre-enforce stages) and Unew.
int set_tables(amss_adjoint* a, double* Unew, double* Z0, double* Z1, double* Z2) {
  for (int t = 0; t < 4; ++t) {
    StepBlock<double>& T = a->host_tab[t];
    T.tl[0] = a->U0;
    T.tl[1] = Unew;
    T.tl[2] = Unew;
    T.K = a->K;
    T.stage[0] = T.stage[1] = nullptr;
  }
  a->host_tab[0].stage[0] = Z0;                                     // sub0: U0 -> A
  a->host_tab[1].stage[0] = a->X[0]; a->host_tab[1].stage[1] = Z1;  // sub1: A -> B
  a->host_tab[2].stage[1] = a->X[1]; a->host_tab[2].stage[0] = Z2;  // sub2: B -> A
  a->host_tab[3].stage[0] = a->X[2];                                // sub3: A -> U_new
  AMSS_CK(cudaMemcpyAsync(a->dtab, a->host_tab, sizeof(a->host_tab), cudaMemcpyHostToDevice, a->stream));
  return 0;
}

// One forward RK4 step: U0raw -> Unew (may alias U0raw: it is read first),
// the pre-enforce stages into Z0..Z2.
// Dsub: where each substep's stencil terms go (null: the scratch a->D).
int fwd_step(amss_adjoint* a, const double* U0raw, double* Unew, double* Z0, double* Z1, double* Z2,
             double* const* Dsub = nullptr) {
  cudaStream_t s = a->stream;
  const long long n = a->npts, fs = a->fs;
  k_enforce_copy<<<grid_of(n), 128, 0, s>>>(U0raw, a->U0, n, fs);
  AMSS_CK(cudaGetLastError());
  double* Z[3] = {Z0, Z1, Z2};
  if (int rc = set_tables(a, Unew, Z0, Z1, Z2)) return rc;
  RKConst rk;
  rk.half_dt = 0.5 * a->dt;
  rk.dt = a->dt;
  rk.sixth_dt = (1.0 / 6.0) * a->dt;
  rk.chitiny = a->chitiny;
  for (int sub = 0; sub < 4; ++sub) {
    const StepBlock<double>* T = a->dtab + sub;
    double* D = Dsub ? Dsub[sub] : a->D;
    AMSS_CK((launch_deriv<double, double>(T, a->ditems, a->nitems, sub, D, a->fs, std::min(a->nitems, 148 * 16), s, 0)));
    AMSS_CK((launch_substep<double, double, false, true, false>(T, a->dtiles, a->ntiles, sub, rk, 0, a->dstatus,
                                                              std::min(a->ntiles, 148 * 8), s, D, a->fs)));
    AMSS_CK((launch_face<double, double, false>(T, a->dfaces, a->nfaces, sub, rk, 0, a->dstatus, s)));
    a->launches += 3;
    if (sub < 3) {
      k_enforce_copy<<<grid_of(n), 128, 0, s>>>(Z[sub], a->X[sub], n, fs);
      AMSS_CK(cudaGetLastError());
      a->launches++;
    }
  }
  return 0;
}

// Xb = F'(X)^T Rb at the input of substep `sub` (table sub), X = input buffer.
// Dpre: X's stencil terms as the forward stored them, or null to recompute.
int rhs_vjp(amss_adjoint* a, int sub, const double* Xin, const double* Rbv, double* Xbv, const double* Dpre) {
  cudaStream_t s = a->stream;
  const StepBlock<double>* T = a->dtab + sub;
  if (!Dpre) {
    AMSS_CK((launch_deriv<double, double>(T, a->ditems, a->nitems, sub, a->D, a->fs, std::min(a->nitems, 148 * 16), s, 0)));
    a->launches++;
  }
  a->host_adj.D = Dpre ? Dpre : a->D;
  a->host_adj.X = Xin;
  a->host_adj.Rb = Rbv;
  a->host_adj.Xb = Xbv;
  AMSS_CK(cudaMemcpyAsync(a->dadj, &a->host_adj, sizeof(AdjBlock), cudaMemcpyHostToDevice, s));
  k_rhs_vjp<<<dim3(grid_of(a->npts), 1), 128, 0, s>>>(a->dadj, a->Db);
  AMSS_CK(cudaGetLastError());
  k_stencil_gather_tiled<<<a->nitems, DTHREADS, kTgSmem, s>>>(a->dadj, a->ditems, a->Db);
  AMSS_CK(cudaGetLastError());
  k_beta_adjoint<<<grid_of(a->npts), 128, 0, s>>>(a->dadj, a->Db);
  AMSS_CK(cudaGetLastError());
  if (a->nfaces) {
    k_face_vjp<<<grid_of(a->nfaces), 128, 0, s>>>(a->dadj, a->dfaces, a->nfaces);
    AMSS_CK(cudaGetLastError());
    a->launches++;
  }
  a->launches += 3;
  return 0;
}

}  // namespace

extern "C" amss_adjoint* amss_adjoint_create(const int ex[3], const double bbox[6], double eps, double chitiny) {
  if (!ex || ex[0] < kDerivMinEx || ex[1] < 7 || ex[2] < 7) {
    amss_fail(AMSS_ERR_ARG, "amss_adjoint_create: needs ex[0] >= 8 and ex[1], ex[2] >= 7");
    return nullptr;
  }
  if ((long long)ex[0] * ex[1] * ex[2] * D_SLOTS >= (1LL << 31) - (1LL << 26)) {
    amss_fail(AMSS_ERR_ARG, "amss_adjoint_create: block too large (the stencil adjoints use 32-bit offsets)");
    return nullptr;
  }
  if (check_device("amss_adjoint_create") != 0) return nullptr;
  if (cudaFuncSetAttribute(k_stencil_gather_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTgSmem) !=
      cudaSuccess) {
    amss_fail(AMSS_ERR_CUDA, "amss_adjoint_create: cannot reserve shared memory for the stencil transpose");
    return nullptr;
  }
  amss_adjoint* a = new amss_adjoint();
  for (int d = 0; d < 3; ++d) a->ex[d] = ex[d];
  a->npts = (long long)ex[0] * ex[1] * ex[2];
  a->fs = pad_stride(a->npts);
  a->eps = eps;
  a->chitiny = chitiny - 1.0;
  std::vector<double> coord(ex[0] + ex[1] + ex[2]);
  double* xs[3] = {coord.data(), coord.data() + ex[0], coord.data() + ex[0] + ex[1]};
  for (int d = 0; d < 3; ++d) {  // Block.C:48-52 (Cell)
    a->dx[d] = (bbox[3 + d] - bbox[d]) / ex[d];
    for (int j = 0; j < ex[d]; ++j) xs[d][j] = bbox[d] + (j + 0.5) * a->dx[d];
  }
  auto fail = [&](const char* m) {
    amss_fail(AMSS_ERR_CUDA, m);
    amss_adjoint_destroy(a);
    return (amss_adjoint*)nullptr;
  };
  const size_t sb = state_bytes(a);
  if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&a->dstatus, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&a->dlvl, 2 * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&a->dcoord, coord.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&a->dtab, sizeof(a->host_tab)) != cudaSuccess ||
      cudaMalloc(&a->dadj, sizeof(AdjBlock)) != cudaSuccess ||
      cudaMalloc(&a->D, (size_t)D_SLOTS * a->fs * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&a->Db, (size_t)D_SLOTS * a->fs * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&a->H, a->fs * sizeof(double)) != cudaSuccess || cudaMalloc(&a->dloss, sizeof(double)) != cudaSuccess)
    return fail("amss_adjoint_create: device allocation failed");
  double** bufs[] = {&a->U, &a->U0, &a->X[0], &a->X[1], &a->X[2], &a->K, &a->Ub, &a->U0b,
                     &a->Rb[0], &a->Rb[1], &a->Rb[2], &a->Rb[3], &a->Xb};
  for (double** b : bufs)
    if (cudaMalloc(b, sb) != cudaSuccess) return fail("amss_adjoint_create: device allocation failed");
  if (cudaMalloc(&a->Zs, 3 * sb) != cudaSuccess) return fail("amss_adjoint_create: device allocation failed");
  cudaMemset(a->dstatus, 0, sizeof(unsigned));
  cudaMemset(a->dlvl, 0, 2 * sizeof(int));
  for (double** b : bufs) cudaMemset(*b, 0, sb);
  cudaMemcpy(a->dcoord, coord.data(), coord.size() * sizeof(double), cudaMemcpyHostToDevice);

  // the block as the engine's kernels see it (level 0, its own patch)
  StepBlock<double> s{};
  s.b.ex[0] = ex[0]; s.b.ex[1] = ex[1]; s.b.ex[2] = ex[2];
  s.b.fs = a->fs;
  s.b.X = a->dcoord; s.b.Y = a->dcoord + ex[0]; s.b.Z = a->dcoord + ex[0] + ex[1];
  s.b.dx[0] = a->dx[0]; s.b.dx[1] = a->dx[1]; s.b.dx[2] = a->dx[2];
  s.b.symmetry = 0;
  block_faces(ex, xs[0], xs[1], xs[2], bbox, 0, &s.b.face_mask, &s.b.lowsym_mask);
  s.C.t = make_coef<double>(s.b.dx, eps);
  s.C.d = s.C.t;
  for (int d = 0; d < 3; ++d) s.d2s[d] = 1.0 / 2.0 / a->dx[d];
  s.lvl = a->dlvl;
  s.doff = 0;
  s.npts = a->npts;
  s.lev0 = 1;
  s.nf = NFIELDS_BSSN;
  s.dw = deriv_tile_w(ex[0]);
  for (int t = 0; t < 4; ++t) a->host_tab[t] = s;
  a->host_adj.b = s.b;
  a->host_adj.C = s.C;
  for (int d = 0; d < 3; ++d) a->host_adj.d2s[d] = s.d2s[d];
  a->host_adj.npts = a->npts;
  a->host_adj.D = a->D;
  a->host_adj.dfs = a->fs;

  std::vector<DerivItem> items;
  std::vector<int2> tiles, faces;
  const int tw = deriv_tile_w(ex[0]), th = deriv_tile_h(ex[0]);
  static const int order[24] = {F_CHI, F_LAP, F_BETAX, F_BETAY, F_BETAZ, F_GXX, F_GXY, F_GXZ,
                                F_GYY, F_GYZ, F_GZZ, F_TRK, F_GAMX, F_GAMY, F_GAMZ, F_AXX,
                                F_AXY, F_AXZ, F_AYY, F_AYZ, F_AZZ, F_DTSFX, F_DTSFY, F_DTSFZ};
  for (int f : order)
    for (int y0 = 0; y0 < ex[1]; y0 += th)
      for (int x0 = 0; x0 < ex[0]; x0 += tw) items.push_back(DerivItem{0, x0, y0, f});
  for (long long p = 0; p < a->npts; p += kPointwiseTile) tiles.push_back(make_int2(0, (int)p));
  const int fm = s.b.face_mask;
  for (int k = 0; k < ex[2]; ++k)
    for (int j = 0; j < ex[1]; ++j)
      for (int i = 0; i < ex[0]; ++i) {
        const bool on = ((fm & 1) && i == ex[0] - 1) || ((fm & 2) && j == ex[1] - 1) || ((fm & 4) && k == ex[2] - 1) ||
                        ((fm & 8) && i == 0) || ((fm & 16) && j == 0) || ((fm & 32) && k == 0);
        if (on) faces.push_back(make_int2(0, (int)(i + (long long)j * ex[0] + (long long)k * ex[0] * ex[1])));
      }
  a->nitems = (int)items.size();
  a->ntiles = (int)tiles.size();
  a->nfaces = (int)faces.size();
  if (cudaMalloc(&a->ditems, items.size() * sizeof(DerivItem)) != cudaSuccess ||
      cudaMalloc(&a->dtiles, tiles.size() * sizeof(int2)) != cudaSuccess ||
      (a->nfaces && cudaMalloc(&a->dfaces, faces.size() * sizeof(int2)) != cudaSuccess))
    return fail("amss_adjoint_create: device allocation failed");
  cudaMemcpy(a->ditems, items.data(), items.size() * sizeof(DerivItem), cudaMemcpyHostToDevice);
  cudaMemcpy(a->dtiles, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice);
  if (a->nfaces) cudaMemcpy(a->dfaces, faces.data(), faces.size() * sizeof(int2), cudaMemcpyHostToDevice);
  return a;
}

extern "C" void amss_adjoint_destroy(amss_adjoint* a) {
  if (!a) return;
  if (a->stream) cudaStreamSynchronize(a->stream);
  void* ptrs[] = {a->dstatus, a->dlvl, a->dcoord, a->dtab, a->dadj, a->ditems, a->dtiles, a->dfaces, a->D, a->Db,
                  a->U, a->U0, a->X[0], a->X[1], a->X[2], a->K, a->Zs, a->H, a->dloss, a->seg, a->Ub, a->U0b,
                  a->Rb[0], a->Rb[1], a->Rb[2], a->Rb[3], a->Xb, a->Dseg};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (double* c : a->ckpt) cudaFree(c);
  if (a->stream) cudaStreamDestroy(a->stream);
  delete a;
}

extern "C" int amss_adjoint_set_state(amss_adjoint* a, const double* h) {
  if (!a || !h) return amss_fail(AMSS_ERR_ARG, "amss_adjoint_set_state: null argument");
  AMSS_CK(cudaMemcpy2DAsync(a->U, a->fs * sizeof(double), h, a->npts * sizeof(double), a->npts * sizeof(double),
                            NFIELDS_BSSN, cudaMemcpyHostToDevice, a->stream));
  AMSS_CK(cudaStreamSynchronize(a->stream));
  a->forward_done = false;
  return 0;
}

extern "C" int amss_adjoint_get_state(amss_adjoint* a, double* h) {
  if (!a || !h) return amss_fail(AMSS_ERR_ARG, "amss_adjoint_get_state: null argument");
  AMSS_CK(cudaMemcpy2DAsync(h, a->npts * sizeof(double), a->U, a->fs * sizeof(double), a->npts * sizeof(double),
                            NFIELDS_BSSN, cudaMemcpyDeviceToHost, a->stream));
  AMSS_CK(cudaStreamSynchronize(a->stream));
  return 0;
}

// The loss of the current a->U and, if want_grad, Ub = dL/dU.
static int loss_and_grad(amss_adjoint* a, double* loss, bool want_grad) {
  cudaStream_t s = a->stream;
  const double dV = a->dx[0] * a->dx[1] * a->dx[2];
  const int gw = 3;
  a->host_tab[0].tl[0] = a->U;   // stencil pass of U (substep-0 input)
  AMSS_CK(cudaMemcpyAsync(a->dtab, a->host_tab, sizeof(StepBlock<double>), cudaMemcpyHostToDevice, s));
  AMSS_CK((launch_deriv<double, double>(a->dtab, a->ditems, a->nitems, 0, a->D, a->fs, std::min(a->nitems, 148 * 16), s, 0)));
  a->host_adj.D = a->D;
  a->host_adj.X = a->U;
  a->host_adj.Rb = nullptr;
  a->host_adj.Xb = a->Ub;
  AMSS_CK(cudaMemcpyAsync(a->dadj, &a->host_adj, sizeof(AdjBlock), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemsetAsync(a->dloss, 0, sizeof(double), s));
  k_ham_loss<<<dim3(grid_of(a->npts), 1), 128, 0, s>>>(a->dadj, gw, dV, a->H, a->dloss);
  AMSS_CK(cudaGetLastError());
  a->launches += 2;
  if (want_grad) {
    AMSS_CK(cudaMemsetAsync(a->Ub, 0, state_bytes(a), s));
    AMSS_CK(cudaMemsetAsync(a->Db, 0, (size_t)D_SLOTS * a->fs * sizeof(double), s));
    k_ham_vjp<<<dim3(grid_of(a->npts), 1), 128, 0, s>>>(a->dadj, gw, dV, a->H, a->Db);
    AMSS_CK(cudaGetLastError());
    k_stencil_gather_tiled<<<a->nitems, DTHREADS, kTgSmem, s>>>(a->dadj, a->ditems, a->Db);   // H reads no adv slot
    AMSS_CK(cudaGetLastError());
    a->launches += 2;
  }
  AMSS_CK(cudaMemcpyAsync(loss, a->dloss, sizeof(double), cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  return 0;
}

// Segment storage: per step U0raw, Z0, Z1, Z2, then the segment's last U_new;
// and, when the device has room for them, the stencil terms of every substep
// of a segment (4 ck arrays of D_SLOTS fields; 92 GB at 96^3 + ghosts with
// ck = 20), so the reverse sweep reads them instead of recomputing them.
static int reserve_segment(amss_adjoint* a) {
  const size_t sb = state_bytes(a);
  const int need = 4 * a->ck + 1;
  if (a->seg_cap < need) {
    if (a->seg) cudaFree(a->seg);
    a->seg = nullptr;
    AMSS_CK(cudaMalloc(&a->seg, (size_t)need * sb));
    a->seg_cap = need;
  }
  const size_t dsz = (size_t)D_SLOTS * a->fs;
  if (a->dseg_cap < 4 * a->ck) {
    if (a->Dseg) cudaFree(a->Dseg);
    a->Dseg = nullptr;
    a->dseg_cap = 0;
    size_t free_b = 0, total_b = 0;
    const size_t want = (size_t)4 * a->ck * dsz * sizeof(double);
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && free_b > want + ((size_t)4 << 30) &&
        cudaMalloc(&a->Dseg, want) == cudaSuccess)
      a->dseg_cap = 4 * a->ck;
    else
      (void)cudaGetLastError();   // not enough room: the reverse sweep recomputes them
  }
  return 0;
}

extern "C" int amss_adjoint_forward(amss_adjoint* a, double dt, int nsteps, int ck, double* loss) {
  if (!a || !loss || nsteps < 0 || ck < 1) return amss_fail(AMSS_ERR_ARG, "amss_adjoint_forward: bad arguments");
  a->dt = dt;
  a->nsteps = nsteps;
  a->ck = ck;
  const size_t sb = state_bytes(a);
  const int nck = (nsteps + ck - 1) / ck;
  if ((int)a->ckpt.size() != nck + 1) {   // + the final state; kept across calls of the same length
    for (double* c : a->ckpt) cudaFree(c);
    a->ckpt.assign(nck + 1, nullptr);
    for (int m = 0; m <= nck; ++m) AMSS_CK(cudaMalloc(&a->ckpt[m], sb));
  }
  a->last_seg_ready = false;
  if (int rc = reserve_segment(a)) return rc;
  cudaStream_t s = a->stream;
  double* Zs1 = a->Zs + (size_t)NFIELDS_BSSN * a->fs;
  double* Zs2 = a->Zs + (size_t)2 * NFIELDS_BSSN * a->fs;
  // the steps of the last segment write their states (and stencil terms)
  // straight into the segment storage, which the reverse sweep starts from
  const long long m = (long long)NFIELDS_BSSN * a->fs;
  const size_t dsz = (size_t)D_SLOTS * a->fs;
  const int nlast = nck > 0 ? (nck - 1) * ck : 0;
  for (int n = 0; n < nsteps; ++n) {
    if (n % ck == 0) AMSS_CK(cudaMemcpyAsync(a->ckpt[n / ck], a->U, sb, cudaMemcpyDeviceToDevice, s));
    if (n >= nlast) {
      const int t = n - nlast;
      double* st0 = a->seg + (size_t)4 * t * m;
      AMSS_CK(cudaMemcpyAsync(st0, a->U, sb, cudaMemcpyDeviceToDevice, s));
      double* const dts[4] = {a->Dseg + (size_t)(4 * t) * dsz, a->Dseg + (size_t)(4 * t + 1) * dsz,
                              a->Dseg + (size_t)(4 * t + 2) * dsz, a->Dseg + (size_t)(4 * t + 3) * dsz};
      if (int rc = fwd_step(a, a->U, a->U, st0 + m, st0 + 2 * m, st0 + 3 * m, a->Dseg ? dts : nullptr)) return rc;
    } else {
      if (int rc = fwd_step(a, a->U, a->U, a->Zs, Zs1, Zs2)) return rc;
    }
  }
  if (nsteps > 0)
    AMSS_CK(cudaMemcpyAsync(a->seg + (size_t)4 * (nsteps - nlast) * m, a->U, sb, cudaMemcpyDeviceToDevice, s));
  AMSS_CK(cudaMemcpyAsync(a->ckpt[nck], a->U, sb, cudaMemcpyDeviceToDevice, s));
  a->last_seg_ready = nsteps > 0;
  if (int rc = loss_and_grad(a, loss, false)) return rc;
  a->forward_done = true;
  return 0;
}

extern "C" int amss_adjoint_backward(amss_adjoint* a, double* grad) {
  if (!a || !grad) return amss_fail(AMSS_ERR_ARG, "amss_adjoint_backward: null argument");
  if (!a->forward_done) return amss_fail(AMSS_ERR_STATE, "amss_adjoint_backward: run amss_adjoint_forward first");
  cudaStream_t s = a->stream;
  const size_t sb = state_bytes(a);
  const long long n = a->npts, fs = a->fs, m = (long long)NFIELDS_BSSN * fs;
  const int nck = (a->nsteps + a->ck - 1) / a->ck;
  if (int rc = reserve_segment(a)) return rc;   // allocated by the forward already
  auto st = [&](int slot) { return a->seg + (size_t)slot * m; };
  const size_t dsz = (size_t)D_SLOTS * fs;
  auto dst = [&](int t, int sub) { return a->Dseg ? a->Dseg + (size_t)(4 * t + sub) * dsz : nullptr; };
  // dL/dU at the final time
  double loss = 0;
  AMSS_CK(cudaMemcpyAsync(a->U, a->ckpt[nck], sb, cudaMemcpyDeviceToDevice, s));
  if (int rc = loss_and_grad(a, &loss, true)) return rc;
  const double dt = a->dt;
  for (int sg = nck - 1; sg >= 0; --sg) {
    const int n0 = sg * a->ck, n1 = std::min(n0 + a->ck, a->nsteps), ns = n1 - n0;
    // recompute the segment, storing what the reverse sweep linearizes about
    // (the last one the forward left in place)
    if (!(sg == nck - 1 && a->last_seg_ready)) {
      AMSS_CK(cudaMemcpyAsync(a->U, a->ckpt[sg], sb, cudaMemcpyDeviceToDevice, s));
      for (int t = 0; t < ns; ++t) {
        AMSS_CK(cudaMemcpyAsync(st(4 * t), a->U, sb, cudaMemcpyDeviceToDevice, s));
        double* const dts[4] = {dst(t, 0), dst(t, 1), dst(t, 2), dst(t, 3)};
        if (int rc = fwd_step(a, a->U, a->U, st(4 * t + 1), st(4 * t + 2), st(4 * t + 3), a->Dseg ? dts : nullptr))
          return rc;
      }
      AMSS_CK(cudaMemcpyAsync(st(4 * ns), a->U, sb, cudaMemcpyDeviceToDevice, s));
    }
    a->last_seg_ready = false;   // the segment storage now holds this segment
    for (int t = ns - 1; t >= 0; --t) {
      double* U0raw = st(4 * t);
      double* Z[3] = {st(4 * t + 1), st(4 * t + 2), st(4 * t + 3)};
      double* Unew = t == ns - 1 ? st(4 * ns) : st(4 * (t + 1));
      // the linearization points: U0 = E(U0raw), X_s = E(Z_{s-1})
      k_enforce_copy<<<grid_of(n), 128, 0, s>>>(U0raw, a->U0, n, fs);
      for (int q = 0; q < 3; ++q) k_enforce_copy<<<grid_of(n), 128, 0, s>>>(Z[q], a->X[q], n, fs);
      AMSS_CK(cudaGetLastError());
      if (int rc = set_tables(a, Unew, Z[0], Z[1], Z[2])) return rc;
      // U_new = floor(U0 + dt/6 (R0 + 2 R1 + 2 R2 + R3))
      k_step_seed<<<grid_of(n), 128, 0, s>>>(a->Ub, Unew, a->U0b, a->Rb[0], a->Rb[1], a->Rb[2], a->Rb[3], dt, n, fs,
                                             a->chitiny);
      AMSS_CK(cudaGetLastError());
      // substeps 3, 2, 1: X_s = E(Z_{s-1}), Z_{s-1} = floor(U0 + c R_{s-1})
      const double c[3] = {0.5 * dt, 0.5 * dt, dt};
      for (int sub = 3; sub >= 1; --sub) {
        if (int rc = rhs_vjp(a, sub, a->X[sub - 1], a->Rb[sub], a->Xb, dst(t, sub))) return rc;
        k_enforce_vjp<true><<<grid_of(n), 128, 0, s>>>(Z[sub - 1], a->Xb, nullptr, nullptr, a->U0b, a->Rb[sub - 1],
                                                 c[sub - 1], n, fs, a->chitiny);
        AMSS_CK(cudaGetLastError());
      }
      if (int rc = rhs_vjp(a, 0, a->U0, a->Rb[0], a->Xb, dst(t, 0))) return rc;
      // the enforce pass at the start of the step: Ub = E'(U0raw)^T (U0b + Xb)
      k_enforce_vjp<false><<<grid_of(n), 128, 0, s>>>(U0raw, a->U0b, a->Xb, a->Ub, nullptr, nullptr, 0.0, n, fs,
                                               a->chitiny);
      AMSS_CK(cudaGetLastError());
      a->launches += 9;
    }
  }
  AMSS_CK(cudaMemcpy2DAsync(grad, n * sizeof(double), a->Ub, fs * sizeof(double), n * sizeof(double), NFIELDS_BSSN,
                            cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  return 0;
}

extern "C" void* amss_adjoint_stream(amss_adjoint* a) { return a ? (void*)a->stream : nullptr; }
extern "C" long long amss_adjoint_launch_count(amss_adjoint* a) { return a ? a->launches : 0; }
