// rhs_noalloc.cu -- compute_rhs_bssn without any device allocation.
//
// Some hosts cannot call cudaMalloc when they evaluate a block's right-hand
// side: a caller running inside a memory pool it does not own, a process whose
// device memory is reserved up front, or a callback that must not fail on
// allocation.  amss_compute_rhs_bssn_noalloc serves them.  It runs the same
// drop-in RHS kernel as compute_rhs_bssn_ (same arguments, same outputs, same
// NaN rule), but its device staging area -- the 24 state fields, 10 matter
// fields, 24 RHS fields, 18 Christoffel symbols, 6 Ricci components, 7
// constraint residuals and the three coordinate lines -- lives in the
// file-scope array below instead of a cudaMalloc'd buffer, and it runs on the
// per-thread default stream instead of a stream it creates.
//
// Limits and sharing:
//   * at most kNoallocMaxPoints = 32768 points per call (e.g. 32^3) and each
//     extent <= kNoallocMaxLine; larger blocks fail with AMSS_ERR_ARG before
//     any device work.  The array is 23.4 MB of device memory per device.
//   * every call uses the same array, which keeps the previous call's
//     contents.  All inputs are copied in and every output point is written by
//     the kernel before it is read back, so only the status word must start at
//     zero; it is cleared on every call.
//   * calls that overlapped on the GPU would race on the array.  The library
//     holds a lock from a call's first copy until its results are back on
//     the host, so calls from the threads of one process run one after the
//     other (another process has its own context and its own copy of the
//     array); a caller must not run the entry point inside a stream capture.
//   * the symbol's device address is looked up once per device context with
//     that device current (cudaGetSymbolAddress), on the first call; a caller
//     that captures work on a stream should make one call first so the lookup
//     is not inside its capture.  The lookup is keyed by the context's unique
//     id (cuCtxGetId), so a caller that resets the device and so gets a new
//     context gets a fresh lookup instead of a stale address.
//   * CUDA loads the library's device code lazily (CUDA_MODULE_LOADING=LAZY,
//     the CUDA 12 default): the first call on a device loads the module and
//     with it allocates this 23.4 MB array.  A host that reserves the rest of
//     the device's memory up front should make its first call before that.
#include <cuda.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "amss_b200.h"
#include "bssn_rhs.cuh"
#include "dev_util.cuh"

namespace amss {

// defined in bssn_kernels.cu / instantiated in rhs_dropin*.cu
template <typename T>
Coef<T> make_coef(const double dx[3], double eps);
void block_faces(const int ex[3], const double* X, const double* Y, const double* Z, const double bbox[6],
                 int symmetry, int* face_mask, int* lowsym_mask);
template <bool SYMM>
cudaError_t launch_rhs_dropin(int grid, cudaStream_t s, BlockView b, Coefs<double> C, const double* u, double* rhs,
                              RhsAux aux, unsigned* status);

constexpr long long kNoallocMaxPoints = AMSS_NOALLOC_MAX_POINTS;
constexpr int kNoallocMaxLine = 4096;
constexpr int kNoallocFields = 24 + 10 + 24 + 18 + 6 + 7;
constexpr long long kNoallocDoubles = kNoallocFields * kNoallocMaxPoints + 3LL * kNoallocMaxLine;

static __device__ __align__(256) double g_noalloc_scratch[kNoallocDoubles];
static __device__ __align__(256) unsigned g_noalloc_status;

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_sym_mu;
double* g_sym_scratch[kMaxDevices] = {};
unsigned* g_sym_status[kMaxDevices] = {};
unsigned long long g_sym_ctx[kMaxDevices] = {};   // id of the context the addresses belong to

// Unique id of the current context (never reused within the process), through
// the driver entry points the runtime hands out; 0 if unavailable.
unsigned long long current_ctx_id() {
  using GetCur = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCur get_cur = nullptr;
  static GetId get_id = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = (GetCur)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (GetId)f;
  }
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_cur && get_id && get_cur(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS) return id;
  return 0;
}

// Device addresses of the scratch array and status word on the current device,
// looked up once per device context (callers hold g_sym_mu).
int noalloc_symbols(double** scratch, unsigned** status) {
  int dev = -1;
  AMSS_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return amss_fail(AMSS_ERR_ARG, "amss_compute_rhs_bssn_noalloc: device index out of range");
  const unsigned long long ctx = current_ctx_id();   // 0 before the runtime made the context current
  if (!g_sym_scratch[dev] || ctx == 0 || ctx != g_sym_ctx[dev]) {
    void* a = nullptr;
    void* b = nullptr;
    AMSS_CK(cudaGetSymbolAddress(&a, g_noalloc_scratch));
    AMSS_CK(cudaGetSymbolAddress(&b, g_noalloc_status));
    g_sym_scratch[dev] = (double*)a;
    g_sym_status[dev] = (unsigned*)b;
    g_sym_ctx[dev] = current_ctx_id();
  }
  *scratch = g_sym_scratch[dev];
  *status = g_sym_status[dev];
  return 0;
}
}  // namespace

}  // namespace amss

using namespace amss;

extern "C" int amss_compute_rhs_bssn_noalloc(
    int* ex, double* T, double* X, double* Y, double* Z, double* chi, double* trK, double* dxx, double* gxy,
    double* gxz, double* dyy, double* gyz, double* dzz, double* Axx, double* Axy, double* Axz, double* Ayy,
    double* Ayz, double* Azz, double* Gamx, double* Gamy, double* Gamz, double* Lap, double* betax, double* betay,
    double* betaz, double* dtSfx, double* dtSfy, double* dtSfz, double* chi_rhs, double* trK_rhs, double* gxx_rhs,
    double* gxy_rhs, double* gxz_rhs, double* gyy_rhs, double* gyz_rhs, double* gzz_rhs, double* Axx_rhs,
    double* Axy_rhs, double* Axz_rhs, double* Ayy_rhs, double* Ayz_rhs, double* Azz_rhs, double* Gamx_rhs,
    double* Gamy_rhs, double* Gamz_rhs, double* Lap_rhs, double* betax_rhs, double* betay_rhs, double* betaz_rhs,
    double* dtSfx_rhs, double* dtSfy_rhs, double* dtSfz_rhs, double* rho, double* Sx, double* Sy, double* Sz,
    double* Sxx, double* Sxy, double* Sxz, double* Syy, double* Syz, double* Szz, double* Gamxxx, double* Gamxxy,
    double* Gamxxz, double* Gamxyy, double* Gamxyz, double* Gamxzz, double* Gamyxx, double* Gamyxy, double* Gamyxz,
    double* Gamyyy, double* Gamyyz, double* Gamyzz, double* Gamzxx, double* Gamzxy, double* Gamzxz, double* Gamzyy,
    double* Gamzyz, double* Gamzzz, double* Rxx, double* Rxy, double* Rxz, double* Ryy, double* Ryz, double* Rzz,
    double* ham_Res, double* movx_Res, double* movy_Res, double* movz_Res, double* Gmx_Res, double* Gmy_Res,
    double* Gmz_Res, int* Symmetry, int* Lev, double* eps, int* co) {
  (void)T;
  (void)Lev;
  if (!ex || ex[0] < 3 || ex[1] < 3 || ex[2] < 3)
    return amss_fail(AMSS_ERR_ARG, "amss_compute_rhs_bssn_noalloc: every extent must be >= 3");
  const long long n = (long long)ex[0] * ex[1] * ex[2];
  if (n > kNoallocMaxPoints || ex[0] > kNoallocMaxLine || ex[1] > kNoallocMaxLine || ex[2] > kNoallocMaxLine) {
    char m[200];
    std::snprintf(m, sizeof m,
                  "amss_compute_rhs_bssn_noalloc: block of %d x %d x %d = %lld points exceeds the static scratch "
                  "limit of %lld points",
                  ex[0], ex[1], ex[2], n, (long long)kNoallocMaxPoints);
    return amss_fail(AMSS_ERR_ARG, m);
  }
  if (check_device("amss_compute_rhs_bssn_noalloc") != 0) return AMSS_ERR_NO_DEVICE;
  double* d = nullptr;
  unsigned* dstatus = nullptr;
  std::lock_guard<std::mutex> lk(g_sym_mu);
  if (int rc = noalloc_symbols(&d, &dstatus)) return rc;

  const long long fs = pad_stride(n);   // <= kNoallocMaxPoints: the limit is a multiple of 64
  double* du = d;
  double* dm = du + 24 * fs;
  double* dr = dm + 10 * fs;
  double* dg = dr + 24 * fs;
  double* dR = dg + 18 * fs;
  double* dc = dR + 6 * fs;
  double* dX = d + kNoallocFields * kNoallocMaxPoints;
  double* dY = dX + kNoallocMaxLine;
  double* dZ = dY + kNoallocMaxLine;
  double* st_in[24] = {chi, trK, dxx, gxy, gxz, dyy, gyz, dzz, Axx, Axy, Axz, Ayy, Ayz, Azz,
                       Gamx, Gamy, Gamz, Lap, betax, betay, betaz, dtSfx, dtSfy, dtSfz};
  double* mat[10] = {rho, Sx, Sy, Sz, Sxx, Sxy, Sxz, Syy, Syz, Szz};
  double* rh[24] = {chi_rhs, trK_rhs, gxx_rhs, gxy_rhs, gxz_rhs, gyy_rhs, gyz_rhs, gzz_rhs,
                    Axx_rhs, Axy_rhs, Axz_rhs, Ayy_rhs, Ayz_rhs, Azz_rhs, Gamx_rhs, Gamy_rhs, Gamz_rhs,
                    Lap_rhs, betax_rhs, betay_rhs, betaz_rhs, dtSfx_rhs, dtSfy_rhs, dtSfz_rhs};
  double* gm[18] = {Gamxxx, Gamxxy, Gamxxz, Gamxyy, Gamxyz, Gamxzz, Gamyxx, Gamyxy, Gamyxz,
                    Gamyyy, Gamyyz, Gamyzz, Gamzxx, Gamzxy, Gamzxz, Gamzyy, Gamzyz, Gamzzz};
  double* rc[6] = {Rxx, Rxy, Rxz, Ryy, Ryz, Rzz};
  double* cs[7] = {ham_Res, movx_Res, movy_Res, movz_Res, Gmx_Res, Gmy_Res, Gmz_Res};
  const size_t bytes = (size_t)n * sizeof(double);
  cudaStream_t s = cudaStreamPerThread;
  for (int f = 0; f < 24; ++f) AMSS_CK(cudaMemcpyAsync(du + f * fs, st_in[f], bytes, cudaMemcpyHostToDevice, s));
  for (int f = 0; f < 10; ++f) AMSS_CK(cudaMemcpyAsync(dm + f * fs, mat[f], bytes, cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dX, X, ex[0] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dY, Y, ex[1] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemcpyAsync(dZ, Z, ex[2] * sizeof(double), cudaMemcpyHostToDevice, s));
  AMSS_CK(cudaMemsetAsync(dstatus, 0, sizeof(unsigned), s));   // the one word that must start at zero

  BlockView b{};
  b.ex[0] = ex[0]; b.ex[1] = ex[1]; b.ex[2] = ex[2];
  b.fs = fs;
  b.X = dX; b.Y = dY; b.Z = dZ;
  b.dx[0] = X[1] - X[0]; b.dx[1] = Y[1] - Y[0]; b.dx[2] = Z[1] - Z[0];
  b.symmetry = *Symmetry;
  {
    const double bb[6] = {X[0], Y[0], Z[0], X[ex[0] - 1], Y[ex[1] - 1], Z[ex[2] - 1]};
    block_faces(ex, X, Y, Z, bb, *Symmetry, &b.face_mask, &b.lowsym_mask);
  }
  Coefs<double> C;
  C.t = make_coef<double>(b.dx, *eps);
  C.d = C.t;
  RhsAux aux{dg, dR, dc, dm, fs, *co};
  long long nb = (n + 127) / 128;
  const int grid = (int)(nb > 148LL * 16 ? 148LL * 16 : nb);
  if (b.lowsym_mask) AMSS_CK(launch_rhs_dropin<true>(grid, s, b, C, du, dr, aux, dstatus));
  else AMSS_CK(launch_rhs_dropin<false>(grid, s, b, C, du, dr, aux, dstatus));
  unsigned hs = 0;
  AMSS_CK(cudaMemcpyAsync(&hs, dstatus, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  if ((hs & ST_NAN) || ((hs & ST_PINF) && (hs & ST_NINF))) return 1;  // bssn_rhs.f90:136, outputs untouched
  for (int f = 0; f < 24; ++f) AMSS_CK(cudaMemcpyAsync(rh[f], dr + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  for (int f = 0; f < 18; ++f) AMSS_CK(cudaMemcpyAsync(gm[f], dg + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  for (int f = 0; f < 6; ++f) AMSS_CK(cudaMemcpyAsync(rc[f], dR + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  if (*co == 0)
    for (int f = 0; f < 7; ++f) AMSS_CK(cudaMemcpyAsync(cs[f], dc + f * fs, bytes, cudaMemcpyDeviceToHost, s));
  AMSS_CK(cudaStreamSynchronize(s));
  return 0;
}
