// engine.cu -- the batched, device-resident evolution engine (amss_engine_*).
//
// All blocks live in one HBM arena.  Per block: the FP64 state U0, two stage
// buffers (FP64, or FP32 in the mixed form), the FP64 RK accumulator K and
// the coordinate arrays.  Per level: a table of StepBlock descriptors and a
// tile list (128 points per tile, tiles never straddle blocks), so one
// persistent launch advances every block of the level, whatever their sizes,
// by one RK4 substep.  Four launches make a step; a step (or many) can be
// captured once as a CUDA graph and replayed.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "bssn_step.cuh"
#include "dev_util.cuh"

namespace amss {

template <typename T>
Coef<T> make_coef(const double dx[3], double eps);
void block_faces(const int ex[3], const double* X, const double* Y, const double* Z, const double bbox[6],
                 int symmetry, int* face_mask, int* lowsym_mask);
template <typename T, typename SS, bool SYMM>
cudaError_t launch_substep(const void* blocks, const int2* tiles, int ntiles, int sub, RKConst rk, int enforce,
                           unsigned* status, int grid, cudaStream_t s);
cudaError_t launch_enforce(long long n, long long fs, double* g, double* a, cudaStream_t s);

static thread_local std::string g_err;

int amss_fail(int code, const char* msg) {
  g_err = msg ? msg : "";
  std::fprintf(stderr, "[amss_b200] %s\n", g_err.c_str());
  return code;
}

int check_device(const char* who) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    char m[256];
    std::snprintf(m, sizeof m,
                  "%s: no usable CUDA device (%s); the B200 kernels have no CPU fallback", who,
                  e != cudaSuccess ? cudaGetErrorString(e) : "device count 0");
    amss_fail(AMSS_ERR_NO_DEVICE, m);
    return -1;
  }
  return 0;
}

struct EBlock {
  int level;
  int ex[3];
  double bbox[6], pbbox[6];
  long long npts, fs;
  std::vector<double> X, Y, Z;
  int face_mask = 0, lowsym = 0;
  double* dX = nullptr;
  double* u0 = nullptr;
  void* st[2] = {nullptr, nullptr};
  double* K = nullptr;
};

struct ELevel {
  std::vector<int> blocks;
  int ntiles = 0;
  int2* dtiles = nullptr;
  void* dtable = nullptr;
  bool symm = false;
};

}  // namespace amss

using namespace amss;

struct amss_engine {
  amss_params prm;
  std::vector<EBlock> blocks;
  std::map<int, ELevel> levels;
  cudaStream_t stream = nullptr;
  unsigned* dstatus = nullptr;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  long long launches = 0;
  bool committed = false;
  int sm_count = 148;
};

extern "C" const char* amss_last_error(void) { return g_err.c_str(); }
extern "C" const char* amss_version(void) { return "amss_b200 0.1 (sm_100a)"; }

extern "C" amss_engine* amss_engine_create(const amss_params* prm) {
  if (!prm) { amss_fail(AMSS_ERR_ARG, "amss_engine_create: null params"); return nullptr; }
  if (check_device("amss_engine_create") != 0) return nullptr;
  amss_engine* e = new amss_engine();
  e->prm = *prm;
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&e->dstatus, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(e->dstatus, 0, sizeof(unsigned)) != cudaSuccess) {
    amss_fail(AMSS_ERR_CUDA, "amss_engine_create: CUDA setup failed");
    delete e;
    return nullptr;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&e->sm_count, cudaDevAttrMultiProcessorCount, dev);
  return e;
}

extern "C" void amss_engine_destroy(amss_engine* e) {
  if (!e) return;
  if (e->stream) cudaStreamSynchronize(e->stream);
  for (auto& kv : e->levels) {
    if (kv.second.dtiles) cudaFree(kv.second.dtiles);
    if (kv.second.dtable) cudaFree(kv.second.dtable);
  }
  if (e->arena) cudaFree(e->arena);
  if (e->dstatus) cudaFree(e->dstatus);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

extern "C" int amss_engine_add_block(amss_engine* e, int level, const int ex[3], const double bbox[6],
                                     const double patch_bbox[6]) {
  if (!e || e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_add_block: engine already committed");
  if (ex[0] < 7 || ex[1] < 7 || ex[2] < 7) return amss_fail(AMSS_ERR_ARG, "amss_engine_add_block: ex < 7");
  EBlock b;
  b.level = level;
  for (int d = 0; d < 3; ++d) b.ex[d] = ex[d];
  for (int m = 0; m < 6; ++m) { b.bbox[m] = bbox[m]; b.pbbox[m] = patch_bbox[m]; }
  b.npts = (long long)ex[0] * ex[1] * ex[2];
  b.fs = pad_stride(b.npts);
  std::vector<double>* xs[3] = {&b.X, &b.Y, &b.Z};
  for (int d = 0; d < 3; ++d) {  // Block.C:48-52 (Cell)
    const double h = (bbox[3 + d] - bbox[d]) / ex[d];
    xs[d]->resize(ex[d]);
    for (int j = 0; j < ex[d]; ++j) (*xs[d])[j] = bbox[d] + (j + 0.5) * h;
  }
  block_faces(b.ex, b.X.data(), b.Y.data(), b.Z.data(), b.pbbox, e->prm.symmetry, &b.face_mask, &b.lowsym);
  e->blocks.push_back(b);
  e->levels[level].blocks.push_back((int)e->blocks.size() - 1);
  return (int)e->blocks.size() - 1;
}

template <typename T>
static int build_table(amss_engine* e, ELevel& L, int level) {
  std::vector<StepBlock<T>> tab;
  std::vector<int2> tiles;
  for (size_t m = 0; m < L.blocks.size(); ++m) {
    EBlock& b = e->blocks[L.blocks[m]];
    StepBlock<T> s{};
    s.b.ex[0] = b.ex[0]; s.b.ex[1] = b.ex[1]; s.b.ex[2] = b.ex[2];
    s.b.fs = b.fs;
    s.b.X = b.dX; s.b.Y = b.dX + b.ex[0]; s.b.Z = b.dX + b.ex[0] + b.ex[1];
    s.b.dx[0] = b.X[1] - b.X[0]; s.b.dx[1] = b.Y[1] - b.Y[0]; s.b.dx[2] = b.Z[1] - b.Z[0];
    s.b.face_mask = b.face_mask;
    s.b.symmetry = e->prm.symmetry;
    s.b.lowsym_mask = b.lowsym;
    s.C = make_coef<T>(s.b.dx, e->prm.eps);
    for (int d = 0; d < 3; ++d) s.d2s[d] = (T)(1.0 / 2.0 / s.b.dx[d]);
    s.u0 = b.u0;
    s.stage[0] = b.st[0];
    s.stage[1] = b.st[1];
    s.K = b.K;
    s.unew = b.u0;
    s.npts = b.npts;
    s.lev0 = level == 0 ? 1 : 0;
    if (b.lowsym) L.symm = true;
    tab.push_back(s);
    for (long long p = 0; p < b.npts; p += 128) tiles.push_back(make_int2((int)m, (int)p));
  }
  L.ntiles = (int)tiles.size();
  AMSS_CK(cudaMalloc(&L.dtable, tab.size() * sizeof(StepBlock<T>)));
  AMSS_CK(cudaMemcpy(L.dtable, tab.data(), tab.size() * sizeof(StepBlock<T>), cudaMemcpyHostToDevice));
  AMSS_CK(cudaMalloc(&L.dtiles, tiles.size() * sizeof(int2)));
  AMSS_CK(cudaMemcpy(L.dtiles, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice));
  return 0;
}

extern "C" int amss_engine_commit(amss_engine* e) {
  if (!e || e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_commit: already committed");
  const bool mixed = e->prm.precision == 1;
  const size_t ss = mixed ? sizeof(float) : sizeof(double);
  size_t bytes = 0;
  auto align = [](size_t x) { return (x + 255) / 256 * 256; };
  for (auto& b : e->blocks) {
    bytes += align((size_t)(b.ex[0] + b.ex[1] + b.ex[2]) * sizeof(double));
    bytes += align((size_t)24 * b.fs * sizeof(double)) * 2;  // u0, K
    bytes += align((size_t)24 * b.fs * ss) * 2;              // two stages
  }
  AMSS_CK(cudaMalloc(&e->arena, bytes));
  AMSS_CK(cudaMemset(e->arena, 0, bytes));
  e->arena_bytes = bytes;
  char* p = e->arena;
  for (auto& b : e->blocks) {
    b.dX = (double*)p;
    p += align((size_t)(b.ex[0] + b.ex[1] + b.ex[2]) * sizeof(double));
    b.u0 = (double*)p; p += align((size_t)24 * b.fs * sizeof(double));
    b.K = (double*)p; p += align((size_t)24 * b.fs * sizeof(double));
    b.st[0] = p; p += align((size_t)24 * b.fs * ss);
    b.st[1] = p; p += align((size_t)24 * b.fs * ss);
    AMSS_CK(cudaMemcpy(b.dX, b.X.data(), b.ex[0] * sizeof(double), cudaMemcpyHostToDevice));
    AMSS_CK(cudaMemcpy(b.dX + b.ex[0], b.Y.data(), b.ex[1] * sizeof(double), cudaMemcpyHostToDevice));
    AMSS_CK(cudaMemcpy(b.dX + b.ex[0] + b.ex[1], b.Z.data(), b.ex[2] * sizeof(double), cudaMemcpyHostToDevice));
  }
  for (auto& kv : e->levels) {
    const int rc = mixed ? build_table<float>(e, kv.second, kv.first) : build_table<double>(e, kv.second, kv.first);
    if (rc) return rc;
  }
  e->committed = true;
  return 0;
}

static int check_block(amss_engine* e, int block) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  if (block < 0 || block >= (int)e->blocks.size()) return amss_fail(AMSS_ERR_ARG, "bad block id");
  return 0;
}

extern "C" int amss_engine_set_state(amss_engine* e, int block, const double* h) {
  if (int rc = check_block(e, block)) return rc;
  EBlock& b = e->blocks[block];
  AMSS_CK(cudaMemcpy2DAsync(b.u0, b.fs * sizeof(double), h, b.npts * sizeof(double), b.npts * sizeof(double), 24,
                            cudaMemcpyHostToDevice, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  return 0;
}

extern "C" int amss_engine_get_state(amss_engine* e, int block, double* h) {
  if (int rc = check_block(e, block)) return rc;
  EBlock& b = e->blocks[block];
  AMSS_CK(cudaMemcpy2DAsync(h, b.npts * sizeof(double), b.u0, b.fs * sizeof(double), b.npts * sizeof(double), 24,
                            cudaMemcpyDeviceToHost, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  return 0;
}

extern "C" int amss_engine_state_device(amss_engine* e, int block, double** dptr, long long* fs) {
  if (int rc = check_block(e, block)) return rc;
  *dptr = e->blocks[block].u0;
  *fs = e->blocks[block].fs;
  return 0;
}

extern "C" int amss_engine_enforce(amss_engine* e) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  for (auto& b : e->blocks) {
    AMSS_CK(launch_enforce(b.npts, b.fs, b.u0 + F_GXX * b.fs, b.u0 + F_AXX * b.fs, e->stream));
    e->launches++;
  }
  return 0;
}

static int step_level_impl(amss_engine* e, int level, double dt) {
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_step_level: no such level");
  ELevel& L = it->second;
  RKConst rk;
  rk.half_dt = 0.5 * dt;
  rk.dt = dt;
  rk.sixth_dt = (1.0 / 6.0) * dt;
  rk.chitiny = e->prm.chitiny;
  const bool mixed = e->prm.precision == 1;
  const int grid = std::min(L.ntiles, e->sm_count * 8);
  for (int sub = 0; sub < 4; ++sub) {
    cudaError_t err;
    if (mixed)
      err = L.symm ? launch_substep<float, float, true>(L.dtable, L.dtiles, L.ntiles, sub, rk, 1, e->dstatus, grid, e->stream)
                   : launch_substep<float, float, false>(L.dtable, L.dtiles, L.ntiles, sub, rk, 1, e->dstatus, grid, e->stream);
    else
      err = L.symm ? launch_substep<double, double, true>(L.dtable, L.dtiles, L.ntiles, sub, rk, 1, e->dstatus, grid, e->stream)
                   : launch_substep<double, double, false>(L.dtable, L.dtiles, L.ntiles, sub, rk, 1, e->dstatus, grid, e->stream);
    AMSS_CK(err);
    e->launches++;
  }
  return 0;
}

extern "C" int amss_engine_step_level(amss_engine* e, int level, double dt) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  return step_level_impl(e, level, dt);
}

extern "C" int amss_engine_run_graph(amss_engine* e, int level, double dt, int nsteps, int replays) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  cudaGraph_t g;
  cudaGraphExec_t ge;
  AMSS_CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  const long long before = e->launches;
  for (int s = 0; s < nsteps; ++s) {
    const int rc = step_level_impl(e, level, dt);
    if (rc) {
      cudaStreamEndCapture(e->stream, &g);
      return rc;
    }
  }
  AMSS_CK(cudaStreamEndCapture(e->stream, &g));
  const long long per_replay = e->launches - before;
  e->launches = before;
  AMSS_CK(cudaGraphInstantiate(&ge, g, 0));
  for (int r = 0; r < replays; ++r) {
    AMSS_CK(cudaGraphLaunch(ge, e->stream));
    e->launches += per_replay;
  }
  AMSS_CK(cudaStreamSynchronize(e->stream));
  cudaGraphExecDestroy(ge);
  cudaGraphDestroy(g);
  return 0;
}

extern "C" int amss_engine_sync(amss_engine* e) {
  if (!e) return AMSS_ERR_ARG;
  AMSS_CK(cudaStreamSynchronize(e->stream));
  unsigned st = 0;
  AMSS_CK(cudaMemcpy(&st, e->dstatus, sizeof(unsigned), cudaMemcpyDeviceToHost));
  return ((st & ST_NAN) || ((st & ST_PINF) && (st & ST_NINF))) ? 1 : 0;
}

extern "C" void* amss_engine_stream(amss_engine* e) { return e ? (void*)e->stream : nullptr; }
extern "C" long long amss_engine_launch_count(amss_engine* e) { return e ? e->launches : 0; }
