// engine.cu -- the batched, device-resident evolution engine (amss_engine_*).
//
// All blocks live in one HBM arena.  Per block: three time levels of the FP64
// state (a ring: current, previous, the one before -- what the reference keeps
// as StateList / OldStateList / SynchList_cor after its rotation,
// bssn_class.C:3852-3853), two stage buffers (FP64, or FP32 plus FP64 chi and
// alpha in the mixed form), the FP64 RK accumulator K and the coordinates.
// The ring is advanced by a one-thread kernel that bumps a per-level index in
// device memory, so kernel arguments never change and a whole Berger-Oliger
// coarse step can be captured once as a CUDA graph and replayed.
//
// Per level: a table of StepBlock descriptors and a tile list (128 points per
// tile, tiles never straddle blocks) so one launch advances every block of the
// level by one RK4 substep; box lists for the same-level ghost sync and, for
// refined levels, for restriction into and prolongation from the parent.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstddef>
#include <map>
#include <string>
#include <vector>

#include "engine_internal.cuh"

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
cudaError_t launch_enforce(long long n, long long fs, double* g, double* a, cudaStream_t s);
template <typename T>
cudaError_t launch_constraints(const void* table, const int2* tiles, int ntiles, int tile_pts, bool symm,
                               const int* region, double* cons, long long dfs, double* part, int grid,
                               cudaStream_t s);
cudaError_t launch_amr_sync(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles, int which,
                            bool fp32_stages, unsigned* status, cudaStream_t s);
cudaError_t launch_amr_prolong(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles,
                               int from_temp, unsigned* status, cudaStream_t s);
cudaError_t launch_amr_restrict(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles,
                                int to_temp, unsigned* status, cudaStream_t s);
cudaError_t launch_amr_timeinterp(const AmrBlock* blocks, const int2* tiles, int ntiles, cudaStream_t s);
cudaError_t launch_amr_timeinterp_boxes(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles,
                                        unsigned* status, cudaStream_t s);
cudaError_t launch_amr_rotate(int* lvl, cudaStream_t s);
cudaError_t launch_amr_enforce(const AmrBlock* blocks, const int2* tiles, int ntiles, cudaStream_t s);
template <typename T>
cudaError_t launch_psi4(const void* table, const int2* tiles, int ntiles, int tile_pts, bool symm, double* scratch,
                        long long dfs, cudaStream_t s);
template <typename T>
cudaError_t launch_admmass(const void* table, const int2* tiles, int ntiles, int tile_pts, bool symm, cudaStream_t s);
void gauss_legendre_desc(int n, std::vector<double>& x, std::vector<double>& w);
double wigner_d(int l, int m, int s, double costheta);

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
    std::snprintf(m, sizeof m, "%s: no usable CUDA device (%s); the B200 kernels have no CPU fallback", who,
                  e != cudaSuccess ? cudaGetErrorString(e) : "device count 0");
    amss_fail(AMSS_ERR_NO_DEVICE, m);
    return -1;
  }
  return 0;
}

}  // namespace amss

using namespace amss;


extern "C" const char* amss_last_error(void) { return g_err.c_str(); }
extern "C" const char* amss_version(void) { return "amss_b200 0.2 (sm_100a)"; }

extern "C" amss_engine* amss_engine_create(const amss_params* prm) {
  if (!prm) { amss_fail(AMSS_ERR_ARG, "amss_engine_create: null params"); return nullptr; }
  if (check_device("amss_engine_create") != 0) return nullptr;
  if (prm->formulation != 0 && prm->formulation != 1) {
    amss_fail(AMSS_ERR_ARG, "amss_engine_create: formulation must be 0 (BSSN) or 1 (Z4c)");
    return nullptr;
  }
  if (prm->formulation == 1 && prm->kernel != 0) {
    amss_fail(AMSS_ERR_UNSUPPORTED, "amss_engine_create: Z4c runs the split kernel form only");
    return nullptr;
  }
  amss_engine* e = new amss_engine();
  e->prm = *prm;
  e->nf = prm->formulation == 1 ? NFIELDS_Z4C : NFIELDS_BSSN;
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&e->dstatus, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(e->dstatus, 0, sizeof(unsigned)) != cudaSuccess) {
    amss_fail(AMSS_ERR_CUDA, "amss_engine_create: CUDA setup failed");
    delete e;
    return nullptr;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  e->device = dev;
  cudaDeviceGetAttribute(&e->sm_count, cudaDevAttrMultiProcessorCount, dev);
  return e;
}

extern "C" void amss_engine_destroy(amss_engine* e) {
  if (!e) return;
  if (e->stream) cudaStreamSynchronize(e->stream);
  amss_xfer_detach(e);
  for (auto& kv : e->levels) {
    ELevel& L = kv.second;
    if (L.dtiles) cudaFree(L.dtiles);
    if (L.dtable) cudaFree(L.dtable);
    if (L.dti_tiles) cudaFree(L.dti_tiles);
    L.dti_boxes.release();
    if (L.ditems) cudaFree(L.ditems);
    if (L.dtiles_f) cudaFree(L.dtiles_f);
    if (L.ditems_f) cudaFree(L.ditems_f);
    if (L.dtiles_s) cudaFree(L.dtiles_s);
    if (L.ditems_s) cudaFree(L.ditems_s);
    if (L.dfaces) cudaFree(L.dfaces);
    if (L.dregion) cudaFree(L.dregion);
    if (L.dregion_first) cudaFree(L.dregion_first);
  }
  release_xfers(e);
  if (e->dblocks) cudaFree(e->dblocks);
  if (e->D) cudaFree(e->D);
  if (e->dlvl) cudaFree(e->dlvl);
  if (e->arena) cudaFree(e->arena);
  if (e->dstatus) cudaFree(e->dstatus);
  if (e->cons) cudaFree(e->cons);
  if (e->cpart) cudaFree(e->cpart);
  if (e->pscr) cudaFree(e->pscr);
  if (e->iitems) cudaFree(e->iitems);
  if (e->dtrack) cudaFree(e->dtrack);
  if (e->dtpatch) cudaFree(e->dtpatch);
  if (e->dtblock) cudaFree(e->dtblock);
  if (e->iout) cudaFree(e->iout);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

static void finish_block(amss_engine* e, EBlock& b, const double bbox[6], const double pbbox[6]) {
  for (int m = 0; m < 6; ++m) { b.bbox[m] = bbox[m]; b.pbbox[m] = pbbox[m]; }
  b.npts = (long long)b.ex[0] * b.ex[1] * b.ex[2];
  b.fs = pad_stride(b.npts);
  std::vector<double>* xs[3] = {&b.X, &b.Y, &b.Z};
  for (int d = 0; d < 3; ++d) {  // Block.C:48-52 (Cell)
    const double h = (bbox[3 + d] - bbox[d]) / b.ex[d];
    xs[d]->resize(b.ex[d]);
    for (int j = 0; j < b.ex[d]; ++j) (*xs[d])[j] = bbox[d] + (j + 0.5) * h;
  }
  block_faces(b.ex, b.X.data(), b.Y.data(), b.Z.data(), b.pbbox, e->prm.symmetry, &b.face_mask, &b.lowsym);
}

extern "C" int amss_engine_add_block(amss_engine* e, int level, const int ex[3], const double bbox[6],
                                     const double patch_bbox[6]) {
  if (!e || e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_add_block: engine already committed");
  if (ex[0] < kDerivMinEx || ex[1] < 7 || ex[2] < 7)
    return amss_fail(AMSS_ERR_ARG, "amss_engine_add_block: needs ex[0] >= 8 and ex[1], ex[2] >= 7");
  EBlock b;
  b.level = level;
  for (int d = 0; d < 3; ++d) {
    b.ex[d] = ex[d];
    b.org[d] = 0;
    b.own.lo[d] = 0;
    b.own.hi[d] = ex[d];
  }
  EPatch p;
  p.level = level;
  p.phys = b.own;
  p.buffer = 0;
  const int pid = (int)e->patches.size();
  p.blocks.push_back((int)e->blocks.size());
  e->patches.push_back(p);
  b.patch = pid;
  b.l2_by_bbox = true;
  finish_block(e, b, bbox, patch_bbox);
  e->blocks.push_back(b);
  e->levels[level].blocks.push_back((int)e->blocks.size() - 1);
  e->levels[level].patches.push_back(pid);
  return (int)e->blocks.size() - 1;
}

extern "C" int amss_engine_set_grid(amss_engine* e, const double x0[3], double h0) {
  if (!e || e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_set_grid: engine already committed");
  if (!(h0 > 0)) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_grid: h0 must be > 0");
  for (int d = 0; d < 3; ++d) e->x0[d] = x0[d];
  e->h0 = h0;
  e->grid_set = true;
  return 0;
}

extern "C" int amss_engine_add_amr_block(amss_engine* e, int level, int patch, const int org[3], const int ex[3],
                                         const int own_lo[3], const int own_hi[3], const int phys_lo[3],
                                         const int phys_hi[3], int buffer) {
  if (!e || e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_add_amr_block: engine already committed");
  if (!e->grid_set) return amss_fail(AMSS_ERR_STATE, "amss_engine_add_amr_block: call amss_engine_set_grid first");
  if (level < 0 || level > 30 || buffer < 0) return amss_fail(AMSS_ERR_ARG, "amss_engine_add_amr_block: bad level/buffer");
  if (ex[0] < kDerivMinEx || ex[1] < 7 || ex[2] < 7)
    return amss_fail(AMSS_ERR_ARG, "amss_engine_add_amr_block: needs ex[0] >= 8 and ex[1], ex[2] >= 7");
  EBlock b;
  b.level = level;
  for (int d = 0; d < 3; ++d) {
    b.ex[d] = ex[d];
    b.org[d] = org[d];
    b.own.lo[d] = own_lo[d];
    b.own.hi[d] = own_hi[d];
    if (ex[d] < 7 || own_lo[d] < org[d] || own_hi[d] > org[d] + ex[d] || own_lo[d] >= own_hi[d])
      return amss_fail(AMSS_ERR_ARG, "amss_engine_add_amr_block: owned box must lie in the array, ex >= 7");
  }
  const auto key = std::make_pair(level, patch);
  auto it = e->patch_ids.find(key);
  int pid;
  if (it == e->patch_ids.end()) {
    EPatch p;
    p.level = level;
    for (int d = 0; d < 3; ++d) { p.phys.lo[d] = phys_lo[d]; p.phys.hi[d] = phys_hi[d]; }
    p.buffer = buffer;
    pid = (int)e->patches.size();
    e->patches.push_back(p);
    e->patch_ids[key] = pid;
    e->levels[level].patches.push_back(pid);
  } else {
    pid = it->second;
  }
  b.patch = pid;
  const double h = e->h0 / std::ldexp(1.0, level);
  const Box ext = e->patches[pid].ext();
  double bbox[6], pbbox[6];
  for (int d = 0; d < 3; ++d) {
    bbox[d] = e->x0[d] + org[d] * h;
    bbox[3 + d] = e->x0[d] + (org[d] + ex[d]) * h;
    pbbox[d] = e->x0[d] + ext.lo[d] * h;
    pbbox[3 + d] = e->x0[d] + ext.hi[d] * h;
  }
  finish_block(e, b, bbox, pbbox);
  e->patches[pid].blocks.push_back((int)e->blocks.size());
  e->blocks.push_back(b);
  e->levels[level].blocks.push_back((int)e->blocks.size() - 1);
  return (int)e->blocks.size() - 1;
}

// Stencil-pass tile width of a block of x extent ex0 on level L: the level's
// tuned width where one is set (at most the block's extent), else deriv_tile_w.
static int level_tile_w(const ELevel& L, int ex0) {
  return L.tile_w > 0 ? std::min(L.tile_w, ex0) : deriv_tile_w(ex0);
}

// Stencil-pass work items of a level: one per (field, x-y tile, z-slab),
// field-major and grouped by stencil kind (the FP64 fields of the mixed form
// first), so resident CTAs of the stencil pass run the same code.  A block's
// z extent is cut into L.zsplit slabs of near-equal height (each slab marches
// its own planes after a 7-plane prologue): more, shorter work items for
// levels whose items would otherwise fill the last wave of CTAs poorly.
// The cells of a block a list covers: 0 its array, 1 its owned cells, 2 its
// final-substep region (global level indices).
static Box list_box(const amss_engine* e, const ELevel& L, const EBlock& b, int mode) {
  if (mode == 1) return intersect(b.own, b.array());
  if (mode == 2) return final_region(e, L, b);
  return b.array();
}

// Stencil-pass work items over each of this rank's blocks of a level: over its
// array (mode 0), its owned cells (1) or its final-substep region (2); x-y tiles
// of the level's tile width, z-slabs, ordered by field.
static std::vector<DerivItem> deriv_items(amss_engine* e, const ELevel& L, int mode = 0) {
  static const int order[25] = {F_CHI, F_LAP, F_BETAX, F_BETAY, F_BETAZ, F_GXX, F_GXY, F_GXZ,
                                F_GYY, F_GYZ, F_GZZ, F_TRK, F_GAMX, F_GAMY, F_GAMZ, F_TZ, F_AXX,
                                F_AXY, F_AXZ, F_AYY, F_AYZ, F_AZZ, F_DTSFX, F_DTSFY, F_DTSFZ};
  std::vector<DerivItem> tiles;
  for (size_t m = 0; m < L.own.size(); ++m) {
    const EBlock& b = e->blocks[L.own[m]];
    if (mode == 0) {
      const int tw = level_tile_w(L, b.ex[0]), th = DTHREADS / tw;
      const int ns = std::max(1, std::min(L.zsplit, b.ex[2] / kMinSlab));
      for (int z = 0; z < ns; ++z) {
        const int k0 = ns == 1 ? 0 : (int)((long long)b.ex[2] * z / ns);
        const int k1 = ns == 1 ? 0 : (int)((long long)b.ex[2] * (z + 1) / ns);
        for (int y0 = 0; y0 < b.ex[1]; y0 += th)
          for (int x0 = 0; x0 < b.ex[0]; x0 += tw) tiles.push_back(DerivItem{(int)m, x0, y0, 0, k0, k1});
      }
      continue;
    }
    const Box r = list_box(e, L, b, mode);
    if (r.empty()) continue;
    int lo[3], n[3];
    for (int d = 0; d < 3; ++d) { lo[d] = r.lo[d] - b.org[d]; n[d] = r.hi[d] - r.lo[d]; }
    // a region narrower than the smallest tile keeps the block's tile, clipped
    const int tw = n[0] >= kDerivMinEx ? level_tile_w(L, n[0]) : level_tile_w(L, b.ex[0]), th = DTHREADS / tw;
    const int ns = std::max(1, std::min(L.zsplit, n[2] / kMinSlab));
    for (int z = 0; z < ns; ++z) {
      const int k0 = lo[2] + (int)((long long)n[2] * z / ns), k1 = lo[2] + (int)((long long)n[2] * (z + 1) / ns);
      for (int y0 = lo[1]; y0 < lo[1] + n[1]; y0 += th)
        for (int x0 = lo[0]; x0 < lo[0] + n[0]; x0 += tw)
          tiles.push_back(DerivItem{(int)m, x0, y0, 0, k0, k1, lo[0] + n[0], lo[1] + n[1], tw});
    }
  }
  std::vector<DerivItem> items;
  for (int f : order) {
    if (f == F_TZ && e->nf != NFIELDS_Z4C) continue;
    for (DerivItem it : tiles) {
      it.field = f;
      items.push_back(it);
    }
  }
  return items;
}

template <typename T>
static int build_table(amss_engine* e, ELevel& L, int level) {
  std::vector<StepBlock<T>> tab;
  std::vector<int2> tiles, tiles_f, tiles_s;
  std::vector<int2> faces;
  std::vector<DerivItem> items;
  long long doff = 0;
  for (size_t m = 0; m < L.own.size(); ++m) {
    EBlock& b = e->blocks[L.own[m]];
    StepBlock<T> s{};
    s.doff = doff;
    doff += b.fs;
    s.b.ex[0] = b.ex[0]; s.b.ex[1] = b.ex[1]; s.b.ex[2] = b.ex[2];
    s.b.fs = b.fs;
    s.b.X = b.dX; s.b.Y = b.dX + b.ex[0]; s.b.Z = b.dX + b.ex[0] + b.ex[1];
    s.b.dx[0] = b.X[1] - b.X[0]; s.b.dx[1] = b.Y[1] - b.Y[0]; s.b.dx[2] = b.Z[1] - b.Z[0];
    s.b.face_mask = b.face_mask;
    s.b.symmetry = e->prm.symmetry;
    s.b.lowsym_mask = b.lowsym;
    s.C.t = make_coef<T>(s.b.dx, e->prm.eps);
    s.C.d = make_coef<double>(s.b.dx, e->prm.eps);
    for (int d = 0; d < 3; ++d) s.d2s[d] = (T)(1.0 / 2.0 / s.b.dx[d]);
    for (int t = 0; t < 3; ++t) s.tl[t] = b.tl[t];
    s.lvl = e->dlvl + 2 * level;
    s.stage[0] = b.st[0];
    s.stage[1] = b.st[1];
    s.side[0] = b.side[0];
    s.side[1] = b.side[1];
    s.K = b.K;
    s.npts = b.npts;
    s.lev0 = level == 0 ? 1 : 0;
    s.nf = e->nf;
    s.dw = level_tile_w(L, b.ex[0]);
    for (int g = 0; g < 2; ++g) {
      const Box r = list_box(e, L, b, g == 0 ? 2 : 1);
      for (int d = 0; d < 3; ++d) {
        s.rlo[g][d] = r.lo[d] - b.org[d];
        s.rn[g][d] = r.empty() ? 0 : r.hi[d] - r.lo[d];
      }
    }
    if (b.lowsym) L.symm = true;
    tab.push_back(s);
    // substep tiles: kPointwiseTile points for the split form's pointwise pass, 128 for the fused kernel
    const long long tstep = e->prm.kernel == 0 ? kPointwiseTile : 128;
    for (long long p = 0; p < b.npts; p += tstep) tiles.push_back(make_int2((int)m, (int)p));
    if (L.final_pad >= 0) {
      const long long nr = (long long)s.rn[0][0] * s.rn[0][1] * s.rn[0][2];
      for (long long q = 0; q < nr; q += tstep) tiles_f.push_back(make_int2((int)m | kRegionTile, (int)q));
    }
    if (L.own_ok) {
      const long long nr = (long long)s.rn[1][0] * s.rn[1][1] * s.rn[1][2];
      for (long long q = 0; q < nr; q += tstep) tiles_s.push_back(make_int2((int)m | kRegionTile | kOwnRegion, (int)q));
    }
    if (b.face_mask) {
      const int fm = b.face_mask;
      for (int k = 0; k < b.ex[2]; ++k)
        for (int j = 0; j < b.ex[1]; ++j)
          for (int i = 0; i < b.ex[0]; ++i) {
            const bool on = ((fm & 1) && i == b.ex[0] - 1) || ((fm & 2) && j == b.ex[1] - 1) ||
                            ((fm & 4) && k == b.ex[2] - 1) || ((fm & 8) && i == 0) || ((fm & 16) && j == 0) ||
                            ((fm & 32) && k == 0);
            if (on) faces.push_back(make_int2((int)m, (int)(i + (long long)j * b.ex[0] + (long long)k * b.ex[0] * b.ex[1])));
          }
    }
  }
  items = deriv_items(e, L);
  const std::vector<DerivItem> items_f = L.final_pad >= 0 ? deriv_items(e, L, 2) : std::vector<DerivItem>();
  const std::vector<DerivItem> items_s = L.own_ok ? deriv_items(e, L, 1) : std::vector<DerivItem>();
  L.ntiles = (int)tiles.size();
  L.ntiles_f = (int)tiles_f.size();
  L.nditems_f = (int)items_f.size();
  L.ntiles_s = (int)tiles_s.size();
  L.nditems_s = (int)items_s.size();
  {
    // constraint-norm region of each table block, in array indices.  A block
    // added by bbox: 3 ghost cells off each side, unless the side's outer cell
    // lies within one cell of the patch box (l2normhelper, fmisc.f90:1286-1303).
    // An AMR block: its owned cells inside its patch, buffer cells included
    // (the patch box of Parallel::L2Norm holds them, MPatch.C:48-51).
    std::vector<int> reg(6 * L.own.size());
    for (size_t m = 0; m < L.own.size(); ++m) {
      const EBlock& b = e->blocks[L.own[m]];
      if (b.l2_by_bbox) {
        const std::vector<double>* xs[3] = {&b.X, &b.Y, &b.Z};
        for (int d = 0; d < 3; ++d) {
          const std::vector<double>& x = *xs[d];
          const double h = x[1] - x[0];
          reg[6 * m + d] = std::fabs(x[0] - b.pbbox[d]) < h ? 0 : 3;
          reg[6 * m + 3 + d] = std::fabs(x[b.ex[d] - 1] - b.pbbox[3 + d]) < h ? b.ex[d] : b.ex[d] - 3;
        }
        continue;
      }
      Box r = intersect(b.own, e->patches[b.patch].ext());
      for (int d = 0; d < 3; ++d) {
        reg[6 * m + d] = r.lo[d] - b.org[d];
        reg[6 * m + 3 + d] = r.hi[d] - b.org[d];
      }
    }
    if (L.dregion) cudaFree(L.dregion);
    if (L.dregion_first) cudaFree(L.dregion_first);
    L.dregion = L.dregion_first = nullptr;
    if (!reg.empty()) {
      AMSS_CK(cudaMalloc(&L.dregion, reg.size() * sizeof(int)));
      AMSS_CK(cudaMemcpy(L.dregion, reg.data(), reg.size() * sizeof(int), cudaMemcpyHostToDevice));
      // the level's first patch (Parallel::L2Norm of GH->PatL[lev]->data, bssn_class.C:7475): the
      // first block's engine patch, or for blocks added by bbox those sharing its patch box
      const EBlock& f0 = e->blocks[L.blocks[0]];
      for (size_t m = 0; m < L.own.size(); ++m) {
        const EBlock& b = e->blocks[L.own[m]];
        const bool first = f0.l2_by_bbox ? (b.l2_by_bbox && std::memcmp(b.pbbox, f0.pbbox, sizeof b.pbbox) == 0)
                                         : b.patch == f0.patch;
        if (!first)
          for (int c = 0; c < 6; ++c) reg[6 * m + c] = 0;
      }
      AMSS_CK(cudaMalloc(&L.dregion_first, reg.size() * sizeof(int)));
      AMSS_CK(cudaMemcpy(L.dregion_first, reg.data(), reg.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
  }
  L.dfs = doff;
  L.nditems = (int)items.size();
  if (tab.empty()) return 0;   // a rank without blocks on this level: no step tables
  AMSS_CK(cudaMalloc(&L.ditems, items.size() * sizeof(DerivItem)));
  AMSS_CK(cudaMemcpy(L.ditems, items.data(), items.size() * sizeof(DerivItem), cudaMemcpyHostToDevice));
  AMSS_CK(cudaMalloc(&L.dtable, tab.size() * sizeof(StepBlock<T>)));
  AMSS_CK(cudaMemcpy(L.dtable, tab.data(), tab.size() * sizeof(StepBlock<T>), cudaMemcpyHostToDevice));
  L.nfaces = (int)faces.size();
  if (!faces.empty()) {
    AMSS_CK(cudaMalloc(&L.dfaces, faces.size() * sizeof(int2)));
    AMSS_CK(cudaMemcpy(L.dfaces, faces.data(), faces.size() * sizeof(int2), cudaMemcpyHostToDevice));
  }
  AMSS_CK(cudaMalloc(&L.dtiles, tiles.size() * sizeof(int2)));
  AMSS_CK(cudaMemcpy(L.dtiles, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice));
  if (!tiles_f.empty()) {
    AMSS_CK(cudaMalloc(&L.dtiles_f, tiles_f.size() * sizeof(int2)));
    AMSS_CK(cudaMemcpy(L.dtiles_f, tiles_f.data(), tiles_f.size() * sizeof(int2), cudaMemcpyHostToDevice));
  }
  if (!items_f.empty()) {
    AMSS_CK(cudaMalloc(&L.ditems_f, items_f.size() * sizeof(DerivItem)));
    AMSS_CK(cudaMemcpy(L.ditems_f, items_f.data(), items_f.size() * sizeof(DerivItem), cudaMemcpyHostToDevice));
  }
  if (!tiles_s.empty()) {
    AMSS_CK(cudaMalloc(&L.dtiles_s, tiles_s.size() * sizeof(int2)));
    AMSS_CK(cudaMemcpy(L.dtiles_s, tiles_s.data(), tiles_s.size() * sizeof(int2), cudaMemcpyHostToDevice));
  }
  if (!items_s.empty()) {
    AMSS_CK(cudaMalloc(&L.ditems_s, items_s.size() * sizeof(DerivItem)));
    AMSS_CK(cudaMemcpy(L.ditems_s, items_s.data(), items_s.size() * sizeof(DerivItem), cudaMemcpyHostToDevice));
  }
  return 0;
}

// Tiles of 128 work units per box: box cells; with nf fields, the (field,
// cell) units the restriction counts, or (runs) the (field, run of
// kProlongRun fine cells along x) units the prolongation counts.
int amss::upload_boxes(const std::vector<AmrBox>& boxes, DevBoxes& D, int nf, bool runs) {
  std::vector<int2> tiles;
  for (size_t m = 0; m < boxes.size(); ++m) {
    const long long nx = runs ? prolong_runs_x(boxes[m].lo[0], boxes[m].n[0]) : boxes[m].n[0];
    const long long n = nx * boxes[m].n[1] * boxes[m].n[2] * (nf ? nf : 1);
    for (long long p = 0; p < n; p += 128) tiles.push_back(make_int2((int)m, (int)p));
  }
  D.ntiles = (int)tiles.size();
  if (boxes.empty()) return 0;
  AMSS_CK(cudaMalloc(&D.boxes, boxes.size() * sizeof(AmrBox)));
  AMSS_CK(cudaMemcpy(D.boxes, boxes.data(), boxes.size() * sizeof(AmrBox), cudaMemcpyHostToDevice));
  AMSS_CK(cudaMalloc(&D.tiles, tiles.size() * sizeof(int2)));
  AMSS_CK(cudaMemcpy(D.tiles, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice));
  return 0;
}

void amss::push_box(std::vector<AmrBox>& v, int dst, int src, const Box& b) {
  if (b.empty()) return;
  AmrBox a;
  a.dst = dst;
  a.src = src;
  for (int d = 0; d < 3; ++d) { a.lo[d] = b.lo[d]; a.n[d] = b.hi[d] - b.lo[d]; }
  v.push_back(a);
}

// Levels 0..L-1 without gaps; each level's owned blocks (every block with one rank).
static int prepare_levels(amss_engine* e, int* nlev_out) {
  int nlev = 0;
  for (auto& kv : e->levels) nlev = std::max(nlev, kv.first + 1);
  for (int l = 0; l < nlev; ++l)
    if (!e->levels.count(l)) return amss_fail(AMSS_ERR_ARG, "amss_engine_commit: levels must be 0..L-1 without gaps");
  for (auto& kv : e->levels) {
    kv.second.own.clear();
    for (int b : kv.second.blocks)
      if (e->owned(b)) kv.second.own.push_back(b);
  }
  *nlev_out = nlev;
  return 0;
}

extern "C" int amss_engine_commit(amss_engine* e) {
  if (!e || e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_commit: already committed");
  if (e->plan_only) return amss_fail(AMSS_ERR_STATE, "amss_engine_commit: a plan-only engine commits with amss_plan_commit");
  if (e->blocks.empty()) return amss_fail(AMSS_ERR_STATE, "amss_engine_commit: no blocks");
  const bool mixed = e->prm.precision == 1;
  const size_t ss = mixed ? sizeof(float) : sizeof(double);
  int nlev = 0;
  if (int rc = prepare_levels(e, &nlev)) return rc;
  if (int rc = build_xfers(e)) return rc;
  plan_final_regions(e);
  // arrays of the blocks this rank owns; the others are geometry only
  size_t bytes = 0;
  auto align = [](size_t x) { return (x + 255) / 256 * 256; };
  for (auto& b : e->blocks) {
    if (b.owner != e->rank) continue;
    bytes += align((size_t)(b.ex[0] + b.ex[1] + b.ex[2]) * sizeof(double));
    bytes += align((size_t)e->nf * b.fs * sizeof(double)) * 4;  // 3 time levels + K
    bytes += align((size_t)e->nf * b.fs * ss) * 2;              // two stages
    if (mixed) bytes += align((size_t)kSideFields * b.fs * sizeof(double)) * 2;
  }
  if (bytes) {
    AMSS_CK(cudaMalloc(&e->arena, bytes));
    AMSS_CK(cudaMemset(e->arena, 0, bytes));
  }
  e->arena_bytes = bytes;
  char* p = e->arena;
  for (auto& b : e->blocks) {
    if (b.owner != e->rank) continue;
    b.dX = (double*)p;
    p += align((size_t)(b.ex[0] + b.ex[1] + b.ex[2]) * sizeof(double));
    for (int t = 0; t < 3; ++t) { b.tl[t] = (double*)p; p += align((size_t)e->nf * b.fs * sizeof(double)); }
    b.K = (double*)p; p += align((size_t)e->nf * b.fs * sizeof(double));
    b.st[0] = p; p += align((size_t)e->nf * b.fs * ss);
    b.st[1] = p; p += align((size_t)e->nf * b.fs * ss);
    if (mixed) {
      b.side[0] = (double*)p; p += align((size_t)kSideFields * b.fs * sizeof(double));
      b.side[1] = (double*)p; p += align((size_t)kSideFields * b.fs * sizeof(double));
    }
    AMSS_CK(cudaMemcpy(b.dX, b.X.data(), b.ex[0] * sizeof(double), cudaMemcpyHostToDevice));
    AMSS_CK(cudaMemcpy(b.dX + b.ex[0], b.Y.data(), b.ex[1] * sizeof(double), cudaMemcpyHostToDevice));
    AMSS_CK(cudaMemcpy(b.dX + b.ex[0] + b.ex[1], b.Z.data(), b.ex[2] * sizeof(double), cudaMemcpyHostToDevice));
  }
  AMSS_CK(cudaMalloc(&e->dlvl, sizeof(int) * 2 * nlev));
  AMSS_CK(cudaMemset(e->dlvl, 0, sizeof(int) * 2 * nlev));
  std::vector<AmrBlock> ab(e->blocks.size());
  for (size_t m = 0; m < e->blocks.size(); ++m) {
    const EBlock& b = e->blocks[m];
    AmrBlock& a = ab[m];
    for (int d = 0; d < 3; ++d) { a.org[d] = b.org[d]; a.ex[d] = b.ex[d]; }
    a.fs = b.fs;
    for (int t = 0; t < 3; ++t) a.tl[t] = b.tl[t];
    a.st[0] = b.st[0]; a.st[1] = b.st[1];
    a.side[0] = b.side[0]; a.side[1] = b.side[1];
    a.K = b.K;
    a.lvl = e->dlvl + 2 * b.level;
    a.nf = e->nf;
  }
  if (int rc = upload_xfers(e, ab)) return rc;   // appends the staging blocks to the table
  AMSS_CK(cudaMalloc(&e->dblocks, ab.size() * sizeof(AmrBlock)));
  AMSS_CK(cudaMemcpy(e->dblocks, ab.data(), ab.size() * sizeof(AmrBlock), cudaMemcpyHostToDevice));
  for (auto& kv : e->levels) {
    ELevel& L = kv.second;
    const int rc = mixed ? build_table<float>(e, L, kv.first) : build_table<double>(e, L, kv.first);
    if (rc) return rc;
    std::vector<int2> ti;
    for (int b : L.own)
      for (long long q = 0; q < e->blocks[b].npts; q += 128) ti.push_back(make_int2(b, (int)q));
    L.nti = (int)ti.size();
    if (!ti.empty()) {
      AMSS_CK(cudaMalloc(&L.dti_tiles, ti.size() * sizeof(int2)));
      AMSS_CK(cudaMemcpy(L.dti_tiles, ti.data(), ti.size() * sizeof(int2), cudaMemcpyHostToDevice));
    }
    if (e->levels.count(kv.first + 1))
      if (int rc = upload_boxes(timeinterp_boxes(e, L, e->levels.at(kv.first + 1)), L.dti_boxes)) return rc;
  }
  if (e->prm.kernel == 0) {
    long long mx = 0;
    for (auto& kv : e->levels) mx = std::max(mx, kv.second.dfs);
    const int slots = e->nf == NFIELDS_Z4C ? D_SLOTS_Z4C : D_SLOTS;
    if (mx) AMSS_CK(cudaMalloc(&e->D, (size_t)mx * slots * (mixed ? sizeof(float) : sizeof(double))));
  }
  if (e->nranks > 1) {
    AMSS_CK(cudaEventCreateWithFlags(&e->ev_ready, cudaEventDisableTiming));
    AMSS_CK(cudaEventCreateWithFlags(&e->ev_done, cudaEventDisableTiming));
  }
  e->committed = true;
  return 0;
}

extern "C" amss_engine* amss_plan_create(const amss_params* prm) {
  if (!prm) { amss_fail(AMSS_ERR_ARG, "amss_plan_create: null params"); return nullptr; }
  if (prm->formulation != 0 && prm->formulation != 1) {
    amss_fail(AMSS_ERR_ARG, "amss_plan_create: formulation must be 0 (BSSN) or 1 (Z4c)");
    return nullptr;
  }
  amss_engine* e = new amss_engine();
  e->prm = *prm;
  e->nf = prm->formulation == 1 ? NFIELDS_Z4C : NFIELDS_BSSN;
  e->plan_only = true;
  return e;
}

extern "C" int amss_plan_commit(amss_engine* e) {
  if (!e || !e->plan_only || e->committed) return amss_fail(AMSS_ERR_STATE, "amss_plan_commit: not an uncommitted plan");
  if (e->blocks.empty()) return amss_fail(AMSS_ERR_STATE, "amss_plan_commit: no blocks");
  int nlev = 0;
  if (int rc = prepare_levels(e, &nlev)) return rc;
  if (int rc = build_xfers(e)) return rc;
  plan_final_regions(e);
  e->committed = true;
  return 0;
}

extern "C" int amss_engine_set_rank(amss_engine* e, int rank, int nranks) {
  if (!e || e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_set_rank: engine already committed");
  if (nranks < 1 || rank < 0 || rank >= nranks) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_rank: need 0 <= rank < nranks");
  e->rank = rank;
  e->nranks = nranks;
  return 0;
}

extern "C" int amss_engine_set_block_owner(amss_engine* e, int block, int owner) {
  if (!e || e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_set_block_owner: engine already committed");
  if (block < 0 || block >= (int)e->blocks.size()) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_block_owner: bad block id");
  if (owner < 0 || owner >= e->nranks) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_block_owner: owner must be 0..nranks-1");
  e->blocks[block].owner = owner;
  return 0;
}

static int check_block(amss_engine* e, int block) {
  if (!e || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  if (block < 0 || block >= (int)e->blocks.size()) return amss_fail(AMSS_ERR_ARG, "bad block id");
  if (!e->owned(block)) return amss_fail(AMSS_ERR_ARG, "block is owned by another rank");
  return 0;
}

// Entry points that need every block on this engine (tracking, point
// interpolation, regrid, graph capture) refuse an engine that holds a share.
static int check_whole(amss_engine* e, const char* who) {
  if (!e || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  if (e->nranks > 1) {
    std::string m = std::string(who) + ": not available on an engine that holds one rank's blocks";
    return amss_fail(AMSS_ERR_UNSUPPORTED, m.c_str());
  }
  return 0;
}

static double* cur_state(amss_engine* e, const EBlock& b) { return b.tl[e->levels[b.level].cur]; }

extern "C" int amss_engine_set_state(amss_engine* e, int block, const double* h) {
  if (int rc = check_block(e, block)) return rc;
  EBlock& b = e->blocks[block];
  AMSS_CK(cudaMemcpy2DAsync(cur_state(e, b), b.fs * sizeof(double), h, b.npts * sizeof(double),
                            b.npts * sizeof(double), e->nf, cudaMemcpyHostToDevice, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  return 0;
}

extern "C" int amss_engine_get_state(amss_engine* e, int block, double* h) {
  if (int rc = check_block(e, block)) return rc;
  EBlock& b = e->blocks[block];
  AMSS_CK(cudaMemcpy2DAsync(h, b.npts * sizeof(double), cur_state(e, b), b.fs * sizeof(double),
                            b.npts * sizeof(double), e->nf, cudaMemcpyDeviceToHost, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  return 0;
}

// The time level `back` steps behind the current state of a block's level (0..2).
static double* time_level(amss_engine* e, const EBlock& b, int back) {
  return b.tl[(e->levels[b.level].cur + 3 - back) % 3];
}

extern "C" int amss_engine_set_time_level(amss_engine* e, int block, int back, const double* h) {
  if (int rc = check_block(e, block)) return rc;
  if (back < 0 || back > 2) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_time_level: back must be 0..2");
  EBlock& b = e->blocks[block];
  AMSS_CK(cudaMemcpy2DAsync(time_level(e, b, back), b.fs * sizeof(double), h, b.npts * sizeof(double),
                            b.npts * sizeof(double), e->nf, cudaMemcpyHostToDevice, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  return 0;
}

extern "C" int amss_engine_get_time_level(amss_engine* e, int block, int back, double* h) {
  if (int rc = check_block(e, block)) return rc;
  if (back < 0 || back > 2) return amss_fail(AMSS_ERR_ARG, "amss_engine_get_time_level: back must be 0..2");
  EBlock& b = e->blocks[block];
  AMSS_CK(cudaMemcpy2DAsync(h, b.npts * sizeof(double), time_level(e, b, back), b.fs * sizeof(double),
                            b.npts * sizeof(double), e->nf, cudaMemcpyDeviceToHost, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  return 0;
}

extern "C" int amss_engine_level_clock(amss_engine* e, int level, int* steps) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_level_clock: no such level");
  if (steps) *steps = (int)it->second.steps;
  return 0;
}

extern "C" int amss_engine_set_level_clock(amss_engine* e, int level, int steps) {
  if (!e || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  auto it = e->levels.find(level);
  if (it == e->levels.end() || steps < 0) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_level_clock: bad level or steps");
  AMSS_CK(cudaStreamSynchronize(e->stream));
  it->second.steps = steps;
  const int st = steps;
  AMSS_CK(cudaMemcpy(e->dlvl + 2 * level + 1, &st, sizeof(int), cudaMemcpyHostToDevice));
  return 0;
}

extern "C" int amss_engine_state_device(amss_engine* e, int block, double** dptr, long long* fs) {
  if (int rc = check_block(e, block)) return rc;
  *dptr = cur_state(e, e->blocks[block]);
  *fs = e->blocks[block].fs;
  return 0;
}

extern "C" int amss_engine_enforce(amss_engine* e) {
  if (!e || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  for (auto& b : e->blocks) {
    if (b.owner != e->rank) continue;
    double* u = cur_state(e, b);
    AMSS_CK(launch_enforce(b.npts, b.fs, u + F_GXX * b.fs, u + F_AXX * b.fs, e->stream));
    e->launches++;
  }
  return 0;
}

static int sync_level(amss_engine* e, ELevel& L, int which) { return run_xfer(e, L.xsync, which); }

// One RK4 step of every block of a level (bssn_class::Step, bssn_class.C:2981-3915):
// four fused substep launches, a ghost sync after each, the ring rotation.
// fin: the step is one of a coarse step, so RestrictProlong follows and the
// final substep may take the level's final-substep regions.
static int step_level_impl(amss_engine* e, int level, double dt, bool fin = false) {
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_step_level: no such level");
  ELevel& L = it->second;
  RKConst rk;
  rk.half_dt = 0.5 * dt;
  rk.dt = dt;
  rk.sixth_dt = (1.0 / 6.0) * dt;
  rk.chitiny = e->prm.chitiny;
  const bool mixed = e->prm.precision == 1;
  // a rank without blocks on this level still takes part in its transfers
  const bool work = !L.own.empty();
  // enforce_ga on U0 in place (bssn_class.C:3052); the stage outputs of
  // substeps 0-2 are enforced as they are written, which equals the
  // reference's in-place enforce_ga at the start of substeps 1-3 (:3416)
  if (work) {
    AMSS_CK(launch_amr_enforce(e->dblocks, L.dti_tiles, L.nti, e->stream));
    e->launches++;
  }
  const bool split = e->prm.kernel == 0;
  const bool track = e->ntrack > 0 && level == e->track_level;
  for (int sub = 0; sub < 4; ++sub) {
    // the final substep over the regions, where the level has them; the
    // others over the owned cells, where the sync after them fills the ghosts
    const bool reg = fin && sub == 3 && L.final_pad >= 0;
    const bool own = !reg && L.own_ok;
    const DerivItem* ditems = reg ? L.ditems_f : own ? L.ditems_s : L.ditems;
    const int nditems = reg ? L.nditems_f : own ? L.nditems_s : L.nditems;
    const int2* tiles = reg ? L.dtiles_f : own ? L.dtiles_s : L.dtiles;
    const int ntiles = reg ? L.ntiles_f : own ? L.ntiles_s : L.ntiles;
    const int dgrid = std::min(nditems, e->sm_count * 16);
    const int grid = std::min(ntiles, e->sm_count * 8);
    if (!work) {
      if (sub < 3)
        if (int rc = sync_level(e, L, sub == 1 ? BUF_STAGE_B : BUF_STAGE_A)) return rc;
      continue;
    }
    cudaError_t err;
    const int enf = sub < 3 ? 1 : 0;
    if (track) {   // the substep's input state is complete (U0, or the synced stage)
      AMSS_CK(launch_track(e->dtpatch, e->ntpatch, e->dtblock, e->dlvl + 2 * level, e->dtrack, e->ntrack, sub, dt,
                           e->prm.symmetry, e->stream));
      e->launches++;
    }
    if (split && nditems) {
      const cudaError_t ed =
          mixed ? launch_deriv<float, float>(L.dtable, ditems, nditems, sub, e->D, L.dfs, dgrid, e->stream, L.docc)
                : launch_deriv<double, double>(L.dtable, ditems, nditems, sub, e->D, L.dfs, dgrid, e->stream, L.docc);
      AMSS_CK(ed);
      e->launches++;
    }
#define AMSS_SUB(T, SY, SP, Z) \
    launch_substep<T, T, SY, SP, Z>(L.dtable, tiles, ntiles, sub, rk, enf, e->dstatus, grid, e->stream, e->D, L.dfs)
    if (ntiles == 0)
      err = cudaSuccess;
    else if (e->nf == NFIELDS_Z4C)   // split form only (checked at create)
      err = mixed ? (L.symm ? AMSS_SUB(float, true, true, true) : AMSS_SUB(float, false, true, true))
                  : (L.symm ? AMSS_SUB(double, true, true, true) : AMSS_SUB(double, false, true, true));
    else if (mixed)
      err = split ? (L.symm ? AMSS_SUB(float, true, true, false) : AMSS_SUB(float, false, true, false))
                  : (L.symm ? AMSS_SUB(float, true, false, false) : AMSS_SUB(float, false, false, false));
    else
      err = split ? (L.symm ? AMSS_SUB(double, true, true, false) : AMSS_SUB(double, false, true, false))
                  : (L.symm ? AMSS_SUB(double, true, false, false) : AMSS_SUB(double, false, false, false));
#undef AMSS_SUB
    AMSS_CK(err);
    if (ntiles) e->launches++;
    // Outer faces.  Level 0: the Sommerfeld rule at every substep.  A refined
    // level's faces are frozen at U0 (enforced in substeps 0-2): the same
    // values in stage A at substeps 0 and 2 and in stage B at substep 1, so
    // substep 0 writes both stages and substeps 1 and 2 launch nothing; the
    // final substep writes the frozen new state unless the level takes
    // regions, past which the faces lie.
    auto face = [&](int s) -> cudaError_t {
      e->launches++;
      return mixed ? (L.symm ? launch_face<float, float, true>(L.dtable, L.dfaces, L.nfaces, s, rk, enf, e->dstatus, e->stream)
                             : launch_face<float, float, false>(L.dtable, L.dfaces, L.nfaces, s, rk, enf, e->dstatus, e->stream))
                   : (L.symm ? launch_face<double, double, true>(L.dtable, L.dfaces, L.nfaces, s, rk, enf, e->dstatus, e->stream)
                             : launch_face<double, double, false>(L.dtable, L.dfaces, L.nfaces, s, rk, enf, e->dstatus, e->stream));
    };
    if (L.nfaces) {
      if (level == 0) {
        AMSS_CK(face(sub));
      } else if (sub == 0) {
        AMSS_CK(face(0));
        AMSS_CK(face(1));
      } else if (sub == 3 && !reg) {
        AMSS_CK(face(3));
      }
    }
    if (sub < 3) {
      if (int rc = sync_level(e, L, sub == 1 ? BUF_STAGE_B : BUF_STAGE_A)) return rc;
    }
  }
  AMSS_CK(launch_amr_rotate(e->dlvl + 2 * level, e->stream));
  e->launches++;
  L.cur = (L.cur + 1) % 3;
  L.steps++;
  return sync_level(e, L, BUF_STATE);
}

// bssn_class::RestrictProlong (bssn_class.C:5724-5903) for level l > 0.
static int restrict_prolong(amss_engine* e, int l, bool same_time) {
  ELevel& F = e->levels[l];
  ELevel& C = e->levels[l - 1];
  if (!same_time && C.dti_boxes.ntiles) {
    // only where the prolongation below reads it
    AMSS_CK(launch_amr_timeinterp_boxes(e->dblocks, C.dti_boxes.boxes, C.dti_boxes.tiles, C.dti_boxes.ntiles,
                                        e->dstatus, e->stream));
    e->launches++;
  }
  const int to_temp = same_time ? 0 : 1;
  if (int rc = run_xfer(e, F.xrestrict, to_temp)) return rc;
  if (int rc = sync_level(e, C, same_time ? BUF_STATE : BUF_TEMP)) return rc;
  if (int rc = run_xfer(e, F.xprolong, to_temp)) return rc;
  return sync_level(e, F, BUF_STATE);
}

// bssn_class::RecursiveStep (bssn_class.C:2323-2414), PSTR 0, RPS 1, trfls 0:
// level 0 takes one step, every finer level two per parent step.
static int recursive_step(amss_engine* e, int l, double dt0) {
  const int nlev = (int)e->levels.size();
  const int iters = l == 0 ? 1 : 2;
  const double dt = dt0 / std::ldexp(1.0, l);
  for (int i = 0; i < iters; ++i) {
    const bool yn = i == iters - 1;
    if (int rc = step_level_impl(e, l, dt, true)) return rc;
    if (l < nlev - 1)
      if (int rc = recursive_step(e, l + 1, dt0)) return rc;
    if (l > 0)
      if (int rc = restrict_prolong(e, l, yn)) return rc;
  }
  return 0;
}

template <typename T>
static int patch_table_dw(amss_engine* e, ELevel& L) {
  for (size_t m = 0; m < L.own.size(); ++m) {
    const int dw = level_tile_w(L, e->blocks[L.own[m]].ex[0]);
    char* dst = (char*)L.dtable + m * sizeof(StepBlock<T>) + offsetof(StepBlock<T>, dw);
    AMSS_CK(cudaMemcpy(dst, &dw, sizeof(int), cudaMemcpyHostToDevice));
  }
  return 0;
}

extern "C" int amss_engine_set_level_tiling(amss_engine* e, int level, int tile_w, int zsplit) {
  if (!e || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_level_tiling: no such level");
  if (tile_w != 0 && (tile_w < kDerivMinEx || tile_w > DWMAX))
    return amss_fail(AMSS_ERR_ARG, "amss_engine_set_level_tiling: tile width must be 0 or 8..64");
  if (zsplit < 1 || zsplit > 16) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_level_tiling: zsplit must be 1..16");
  ELevel& L = it->second;
  AMSS_CK(cudaStreamSynchronize(e->stream));
  L.tile_w = tile_w;
  L.zsplit = zsplit;
  const std::vector<DerivItem> items = deriv_items(e, L);
  const std::vector<DerivItem> items_f = L.final_pad >= 0 ? deriv_items(e, L, 2) : std::vector<DerivItem>();
  const std::vector<DerivItem> items_s = L.own_ok ? deriv_items(e, L, 1) : std::vector<DerivItem>();
  if (L.ditems) cudaFree(L.ditems);
  if (L.ditems_f) cudaFree(L.ditems_f);
  if (L.ditems_s) cudaFree(L.ditems_s);
  L.ditems = L.ditems_f = L.ditems_s = nullptr;
  L.nditems = (int)items.size();
  L.nditems_f = (int)items_f.size();
  L.nditems_s = (int)items_s.size();
  if (items.empty()) return 0;
  AMSS_CK(cudaMalloc(&L.ditems, items.size() * sizeof(DerivItem)));
  AMSS_CK(cudaMemcpy(L.ditems, items.data(), items.size() * sizeof(DerivItem), cudaMemcpyHostToDevice));
  if (!items_f.empty()) {
    AMSS_CK(cudaMalloc(&L.ditems_f, items_f.size() * sizeof(DerivItem)));
    AMSS_CK(cudaMemcpy(L.ditems_f, items_f.data(), items_f.size() * sizeof(DerivItem), cudaMemcpyHostToDevice));
  }
  if (!items_s.empty()) {
    AMSS_CK(cudaMalloc(&L.ditems_s, items_s.size() * sizeof(DerivItem)));
    AMSS_CK(cudaMemcpy(L.ditems_s, items_s.data(), items_s.size() * sizeof(DerivItem), cudaMemcpyHostToDevice));
  }
  return e->prm.precision == 1 ? patch_table_dw<float>(e, L) : patch_table_dw<double>(e, L);
}

extern "C" int amss_engine_level_final_region(amss_engine* e, int level, int* pad, long long* points) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_level_final_region: no such level");
  const ELevel& L = it->second;
  if (pad) *pad = L.final_pad;
  if (points) {
    long long n = 0;
    const int mode = L.final_pad >= 0 ? 2 : L.own_ok ? 1 : 0;
    for (int b : L.own) {
      const Box r = list_box(e, L, e->blocks[b], mode);
      if (!r.empty()) n += (long long)(r.hi[0] - r.lo[0]) * (r.hi[1] - r.lo[1]) * (r.hi[2] - r.lo[2]);
    }
    *points = n;
  }
  return 0;
}

extern "C" int amss_engine_set_level_occupancy(amss_engine* e, int level, int occ) {
  if (!e || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_level_occupancy: no such level");
  if (occ != 0 && occ != 1) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_level_occupancy: occupancy 0 or 1");
  it->second.docc = occ;
  return 0;
}

extern "C" int amss_engine_get_level_occupancy(amss_engine* e, int level, int* occ) {
  if (!e || !e->committed || !occ) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_get_level_occupancy: no such level");
  *occ = it->second.docc;
  return 0;
}

extern "C" int amss_engine_get_level_tiling(amss_engine* e, int level, int* tile_w, int* zsplit, int* nitems) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_get_level_tiling: no such level");
  if (tile_w) *tile_w = it->second.tile_w;
  if (zsplit) *zsplit = it->second.zsplit;
  if (nitems) *nitems = it->second.nditems;
  return 0;
}

// ---- regrid: fill a level of a new hierarchy from the engine it replaces ----

// a \ b as disjoint boxes
static void box_subtract(const Box& a, const Box& b, std::vector<Box>& out) {
  const Box i = intersect(a, b);
  if (i.empty()) { out.push_back(a); return; }
  Box rest = a;
  for (int d = 0; d < 3; ++d) {
    if (rest.lo[d] < i.lo[d]) { Box s = rest; s.hi[d] = i.lo[d]; out.push_back(s); rest.lo[d] = i.lo[d]; }
    if (i.hi[d] < rest.hi[d]) { Box s = rest; s.lo[d] = i.hi[d]; out.push_back(s); rest.hi[d] = i.hi[d]; }
  }
}

// The AMR kernels' view of a block; its current state slot is tl[*lvl], so
// the time level `back` steps behind the current one is presented by
// rotating the ring (cur = the level's host mirror).
static AmrBlock amr_view(const amss_engine* e, const EBlock& b, int cur, int back) {
  AmrBlock a{};
  for (int d = 0; d < 3; ++d) { a.org[d] = b.org[d]; a.ex[d] = b.ex[d]; }
  a.fs = b.fs;
  for (int t = 0; t < 3; ++t) a.tl[t] = b.tl[t];
  a.tl[cur] = b.tl[(cur + 3 - back) % 3];
  a.st[0] = b.st[0]; a.st[1] = b.st[1];
  a.side[0] = b.side[0]; a.side[1] = b.side[1];
  a.K = b.K;
  a.lvl = e->dlvl + 2 * b.level;
  a.nf = e->nf;
  return a;
}

extern "C" int amss_engine_regrid_fill(amss_engine* dst, amss_engine* src, int level, int back) {
  if (!dst || !src || !dst->committed || !src->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  if (int rc = check_whole(dst, "amss_engine_regrid_fill")) return rc;
  if (int rc = check_whole(src, "amss_engine_regrid_fill")) return rc;
  if (dst == src) return amss_fail(AMSS_ERR_ARG, "amss_engine_regrid_fill: source and destination are one engine");
  if (back != 0 && back != 1) return amss_fail(AMSS_ERR_ARG, "amss_engine_regrid_fill: back must be 0 or 1");
  if (dst->nf != src->nf || dst->prm.precision != src->prm.precision)
    return amss_fail(AMSS_ERR_ARG, "amss_engine_regrid_fill: engines differ in fields or precision");
  for (int d = 0; d < 3; ++d)
    if (dst->x0[d] != src->x0[d]) return amss_fail(AMSS_ERR_ARG, "amss_engine_regrid_fill: grids differ");
  if (dst->h0 != src->h0) return amss_fail(AMSS_ERR_ARG, "amss_engine_regrid_fill: grids differ");
  auto id = dst->levels.find(level), is = src->levels.find(level);
  if (id == dst->levels.end() || is == src->levels.end())
    return amss_fail(AMSS_ERR_ARG, "amss_engine_regrid_fill: level missing in one engine");
  ELevel& LD = id->second;
  ELevel& LS = is->second;
  AMSS_CK(cudaStreamSynchronize(src->stream));
  AMSS_CK(cudaStreamSynchronize(dst->stream));
  // the level keeps its clock (ring index, steps taken)
  AMSS_CK(cudaMemcpy(dst->dlvl + 2 * level, src->dlvl + 2 * level, 2 * sizeof(int), cudaMemcpyDeviceToDevice));
  LD.cur = LS.cur;
  LD.steps = LS.steps;
  // table: the destination level's blocks, the source level's, the source parent's
  std::vector<AmrBlock> tab;
  for (int b : LD.blocks) tab.push_back(amr_view(dst, dst->blocks[b], LD.cur, back));
  for (int b : LS.blocks) tab.push_back(amr_view(src, src->blocks[b], LS.cur, back));
  const ELevel* LP = nullptr;
  if (level > 0) {
    LP = &src->levels[level - 1];
    for (int b : LP->blocks) tab.push_back(amr_view(src, src->blocks[b], LP->cur, 0));
  }
  const int nD = (int)LD.blocks.size(), nS = (int)LS.blocks.size();
  // copy: every destination cell (ghosts included) that a source block owns
  std::vector<AmrBox> cp, pr;
  for (int i = 0; i < nD; ++i)
    for (int j = 0; j < nS; ++j)
      push_box(cp, i, nD + j, intersect(dst->blocks[LD.blocks[i]].array(), src->blocks[LS.blocks[j]].own));
  // prolong: destination cells outside every source patch (buffers included),
  // from the source parent block that owns their parent cell
  for (int i = 0; i < nD; ++i) {
    std::vector<Box> pieces{dst->blocks[LD.blocks[i]].array()};
    for (int pid : LS.patches) {
      std::vector<Box> next;
      for (const Box& q : pieces) box_subtract(q, src->patches[pid].ext(), next);
      pieces.swap(next);
    }
    for (const Box& q : pieces) {
      if (!LP) return amss_fail(AMSS_ERR_ARG, "amss_engine_regrid_fill: level 0 must keep its extent");
      for (size_t c = 0; c < LP->blocks.size(); ++c) {
        const Box& o = src->blocks[LP->blocks[c]].own;
        Box of;
        for (int d = 0; d < 3; ++d) { of.lo[d] = 2 * o.lo[d]; of.hi[d] = 2 * o.hi[d]; }
        push_box(pr, i, nD + nS + (int)c, intersect(q, of));
      }
    }
  }
  AmrBlock* dtab = nullptr;
  DevBoxes dcp, dpr;
  int rc = 0;
  unsigned hs = 0;
  AMSS_CK(cudaMalloc(&dtab, tab.size() * sizeof(AmrBlock)));
  AMSS_CK(cudaMemcpy(dtab, tab.data(), tab.size() * sizeof(AmrBlock), cudaMemcpyHostToDevice));
  AMSS_CK(cudaMemsetAsync(dst->dstatus, 0, sizeof(unsigned), dst->stream));
  if ((rc = upload_boxes(cp, dcp)) == 0 && (rc = upload_boxes(pr, dpr, dst->nf, true)) == 0) {
    cudaError_t err = cudaSuccess;
    if (dcp.ntiles)
      err = launch_amr_sync(dtab, dcp.boxes, dcp.tiles, dcp.ntiles, BUF_STATE, dst->prm.precision == 1, dst->dstatus,
                            dst->stream);
    if (err == cudaSuccess && dpr.ntiles && back == 1)   // the parent between its current and previous levels
      err = launch_amr_timeinterp(src->dblocks, LP->dti_tiles, LP->nti, dst->stream);
    if (err == cudaSuccess && dpr.ntiles)
      err = launch_amr_prolong(dtab, dpr.boxes, dpr.tiles, dpr.ntiles, back, dst->dstatus, dst->stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&hs, dst->dstatus, sizeof(unsigned), cudaMemcpyDeviceToHost, dst->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(dst->stream);
    if (err != cudaSuccess) rc = amss_fail(AMSS_ERR_CUDA, cudaGetErrorString(err));
  }
  dcp.release();
  dpr.release();
  cudaFree(dtab);
  if (rc) return rc;
  if (hs & ST_BAD_ARG)
    return amss_fail(AMSS_ERR_ARG, "amss_engine_regrid_fill: a cell to fill lies outside the source's parent blocks "
                                   "(the new boxes are not nested in the old parent level)");
  return 0;
}

extern "C" int amss_engine_step_level(amss_engine* e, int level, double dt) {
  if (!e || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  if (e->nranks > 1) AMSS_CK(cudaSetDevice(e->device));   // each rank's thread drives its own GPU
  return step_level_impl(e, level, dt);
}

extern "C" int amss_engine_coarse_step(amss_engine* e, double dt0) {
  if (!e || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  if (e->nranks > 1) AMSS_CK(cudaSetDevice(e->device));   // each rank's thread drives its own GPU
  return recursive_step(e, 0, dt0);
}

// Capture `nsteps` of either a single-level step (level >= 0) or a coarse
// Berger-Oliger step (level < 0) once as a graph and replay it.
static int run_graph(amss_engine* e, int level, double dt, int nsteps, int replays) {
  cudaGraph_t g;
  cudaGraphExec_t ge;
  std::vector<int> cur0;
  std::vector<long long> steps0;
  for (auto& kv : e->levels) { cur0.push_back(kv.second.cur); steps0.push_back(kv.second.steps); }
  const long long before = e->launches;
  AMSS_CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  int rc = 0;
  for (int s = 0; s < nsteps && rc == 0; ++s) rc = level >= 0 ? step_level_impl(e, level, dt) : recursive_step(e, 0, dt);
  cudaError_t ec = cudaStreamEndCapture(e->stream, &g);
  if (rc) return rc;
  AMSS_CK(ec);
  const long long per_replay = e->launches - before;
  // capture issued nothing yet: undo the host mirrors and re-advance them per replay
  std::vector<int> dcur;
  std::vector<long long> dsteps;
  size_t q = 0;
  for (auto& kv : e->levels) {
    dcur.push_back(((kv.second.cur - cur0[q]) % 3 + 3) % 3);
    dsteps.push_back(kv.second.steps - steps0[q]);
    kv.second.cur = cur0[q];
    kv.second.steps = steps0[q];
    ++q;
  }
  e->launches = before;
  AMSS_CK(cudaGraphInstantiate(&ge, g, 0));
  for (int r = 0; r < replays; ++r) {
    AMSS_CK(cudaGraphLaunch(ge, e->stream));
    e->launches += per_replay;
    q = 0;
    for (auto& kv : e->levels) {
      kv.second.cur = (kv.second.cur + dcur[q]) % 3;
      kv.second.steps += dsteps[q];
      ++q;
    }
  }
  AMSS_CK(cudaStreamSynchronize(e->stream));
  cudaGraphExecDestroy(ge);
  cudaGraphDestroy(g);
  return 0;
}

extern "C" int amss_engine_run_graph(amss_engine* e, int level, double dt, int nsteps, int replays) {
  if (int rc = check_whole(e, "amss_engine_run_graph")) return rc;
  if (level < 0) return amss_fail(AMSS_ERR_ARG, "amss_engine_run_graph: level must be >= 0");
  return run_graph(e, level, dt, nsteps, replays);
}

extern "C" int amss_engine_run_coarse_graph(amss_engine* e, double dt0, int nsteps, int replays) {
  if (int rc = check_whole(e, "amss_engine_run_coarse_graph")) return rc;
  return run_graph(e, -1, dt0, nsteps, replays);
}

extern "C" int amss_engine_sync(amss_engine* e) {
  if (!e) return AMSS_ERR_ARG;
  if (e->plan_only) return amss_fail(AMSS_ERR_STATE, "amss_engine_sync: a plan has no device state");
  AMSS_CK(cudaStreamSynchronize(e->stream));
  unsigned st = 0;
  AMSS_CK(cudaMemcpy(&st, e->dstatus, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (st & ST_BAD_ARG) return amss_fail(AMSS_ERR_STATE, "a kernel met a box outside its block (engine tables)");
  if (st & ST_TIMEOUT) return amss_fail(AMSS_ERR_CUDA, "a bounded wait on an asynchronous copy gave up");
  return ((st & ST_NAN) || ((st & ST_PINF) && (st & ST_NINF))) ? 1 : 0;
}

extern "C" void* amss_engine_stream(amss_engine* e) { return e ? (void*)e->stream : nullptr; }
extern "C" long long amss_engine_launch_count(amss_engine* e) { return e ? e->launches : 0; }

extern "C" long long amss_engine_level_points(amss_engine* e, int level) {
  if (!e) return -1;
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return 0;
  long long n = 0;
  for (int b : it->second.own) n += e->blocks[b].npts;
  return n;
}

static int constraint_sums(amss_engine* e, int level, double* sums, bool first_patch);

extern "C" int amss_engine_constraint_sums(amss_engine* e, int level, double* sums) {
  return constraint_sums(e, level, sums, false);
}

extern "C" int amss_engine_constraint_norms_first_patch(amss_engine* e, int level, double* norms) {
  if (!norms) return amss_fail(AMSS_ERR_ARG, "amss_engine_constraint_norms_first_patch: null argument");
  double s[8];
  if (int rc = constraint_sums(e, level, s, true)) return rc;
  for (int c = 0; c < 8; ++c) norms[c] = std::sqrt(s[c]);
  return 0;
}

static int constraint_sums(amss_engine* e, int level, double* sums, bool first_patch) {
  if (!e || !sums) return amss_fail(AMSS_ERR_ARG, "amss_engine_constraint_sums: null argument");
  if (!e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "amss_engine_constraint_sums: commit the engine first");
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_constraint_sums: no such level");
  ELevel& L = it->second;
  if (L.own.empty()) {   // a rank without blocks on the level adds nothing
    for (int c = 0; c < 8; ++c) sums[c] = 0.0;
    return 0;
  }
  constexpr int kGrid = 148 * 2;
  if (e->cons_cap < 7 * L.dfs) {
    if (e->cons) cudaFree(e->cons);
    e->cons = nullptr;
    e->cons_cap = 0;
    AMSS_CK(cudaMalloc(&e->cons, (size_t)7 * L.dfs * sizeof(double)));
    e->cons_cap = 7 * L.dfs;
  }
  if (!e->cpart) AMSS_CK(cudaMalloc(&e->cpart, (size_t)kGrid * 8 * sizeof(double)));
  const int tile_pts = e->prm.kernel == 0 ? (int)kPointwiseTile : 128;
  const cudaError_t err =
      e->prm.precision == 1
          ? launch_constraints<float>(L.dtable, L.dtiles, L.ntiles, tile_pts, L.symm,
                                      first_patch ? L.dregion_first : L.dregion, e->cons, L.dfs, e->cpart, kGrid,
                                      e->stream)
          : launch_constraints<double>(L.dtable, L.dtiles, L.ntiles, tile_pts, L.symm,
                                       first_patch ? L.dregion_first : L.dregion, e->cons, L.dfs, e->cpart, kGrid,
                                       e->stream);
  AMSS_CK(err);
  e->launches += 2;
  std::vector<double> part((size_t)kGrid * 8);
  AMSS_CK(cudaMemcpyAsync(part.data(), e->cpart, part.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  for (int c = 0; c < 8; ++c) {
    double v = 0.0;
    for (int g = 0; g < kGrid; ++g) v += part[(size_t)g * 8 + c];   // fixed order: reproducible
    sums[c] = v;
  }
  return 0;
}

extern "C" int amss_engine_constraint_norms(amss_engine* e, int level, double* norms) {
  if (!norms) return amss_fail(AMSS_ERR_ARG, "amss_engine_constraint_norms: null argument");
  double s[8];
  if (int rc = amss_engine_constraint_sums(e, level, s)) return rc;
  for (int c = 0; c < 8; ++c) norms[c] = std::sqrt(s[c]);
  return 0;
}

// The patches of a level as Parallel::PatList_Interp_Points walks them:
// engine patches in order; blocks added by bbox grouped by their patch box.
struct IPatch {
  int patch;           // engine patch, -1 for a group of blocks added by bbox
  double pbb[6], h[3];
  int buffer;
  std::vector<int> blocks;
};

static std::vector<IPatch> level_patches(amss_engine* e, const ELevel& L) {
  std::vector<IPatch> ps;
  for (int bid : L.blocks) {
    const EBlock& b = e->blocks[bid];
    IPatch* g = nullptr;
    for (auto& q : ps)
      if ((b.l2_by_bbox && q.patch < 0 && std::memcmp(q.pbb, b.pbbox, sizeof q.pbb) == 0) ||
          (!b.l2_by_bbox && q.patch == b.patch))
        g = &q;
    if (!g) {
      IPatch q;
      q.patch = b.l2_by_bbox ? -1 : b.patch;
      std::memcpy(q.pbb, b.pbbox, sizeof q.pbb);
      q.buffer = b.l2_by_bbox ? 0 : e->patches[b.patch].buffer;
      for (int d = 0; d < 3; ++d) {
        long long shape;
        if (b.l2_by_bbox) {
          const double hb = (b.bbox[3 + d] - b.bbox[d]) / b.ex[d];
          shape = std::llround((b.pbbox[3 + d] - b.pbbox[d]) / hb);
        } else {
          const Box x = e->patches[b.patch].ext();
          shape = x.hi[d] - x.lo[d];
        }
        q.h[d] = (q.pbb[3 + d] - q.pbb[d]) / (double)shape;   // Patch::getdX
      }
      ps.push_back(q);
      g = &ps.back();
    }
    g->blocks.push_back(bid);
  }
  return ps;
}

// Patch::Interp_Points' box of a block (Cell): less the buffer on a side it
// shares with the patch box, else less the ghosts.
static void find_box(const EBlock& b, const IPatch& q, double lo[3], double hi[3]) {
  for (int d = 0; d < 3; ++d) {
    const double h = q.h[d];
    lo[d] = std::fabs(b.bbox[d] - q.pbb[d]) < h / 2 ? b.bbox[d] + q.buffer * h : b.bbox[d] + 3 * h;
    hi[d] = std::fabs(b.bbox[3 + d] - q.pbb[3 + d]) < h / 2 ? b.bbox[3 + d] - q.buffer * h : b.bbox[3 + d] - 3 * h;
  }
}

// Point interpolation on a level.  Host side of Parallel::PatList_Interp_Points
// (Parallel.C:5614-5667) and Patch::Interp_Points (MPatch.C:339-500, Cell):
// the first patch of the level whose box less its buffer holds the point, then
// the first block of that patch whose box less its ghosts (less the buffer on
// a side it shares with the patch box) holds it to half a cell; and the
// stencil choice of global_interp (fmisc.f90:738-781, ORDN = 6).  Blocks added
// by bbox form one patch per distinct patch box, with no buffer.
// from_acc: the fields are those of the blocks' accumulators K (Psi4 after
// amss_engine_psi4) instead of the current state.
static int interp_level(amss_engine* e, int level, int npts, const double* xyz, int nvar, const int* fields,
                        const double* soa, double* out, int* found, bool from_acc) {
  if (!e || (npts > 0 && (!xyz || !out)) || nvar < 1 || !fields)
    return amss_fail(AMSS_ERR_ARG, "amss_engine_interp_points: null argument or nvar < 1");
  if (!e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_interp_points: commit the engine first");
  if (int rc = check_whole(e, "amss_engine_interp_points")) return rc;
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_interp_points: no such level");
  for (int v = 0; v < nvar; ++v)
    if (fields[v] < 0 || fields[v] >= e->nf) return amss_fail(AMSS_ERR_ARG, "amss_engine_interp_points: bad field");
  if (npts <= 0) return 0;
  const std::vector<IPatch> ps = level_patches(e, it->second);
  std::vector<InterpItem> items;
  std::vector<long long> where;   // output slot of each item
  for (int p = 0; p < npts; ++p) {
    const double* pt = xyz + 3 * (long long)p;
    if (!std::isfinite(pt[0]) || !std::isfinite(pt[1]) || !std::isfinite(pt[2]))
      return amss_fail(AMSS_ERR_ARG, "amss_engine_interp_points: a point is not finite");
    int ok = 0;
    for (const auto& q : ps) {
      bool inp = true;
      for (int d = 0; d < 3; ++d)
        if (pt[d] < q.pbb[d] + q.buffer * q.h[d] || pt[d] > q.pbb[3 + d] - q.buffer * q.h[d]) inp = false;
      if (!inp) continue;
      for (int bid : q.blocks) {
        const EBlock& b = e->blocks[bid];
        bool inb = true;
        double lo[3], hi[3];
        find_box(b, q, lo, hi);
        for (int d = 0; d < 3; ++d)
          if (pt[d] - lo[d] < -q.h[d] / 2 || pt[d] - hi[d] > q.h[d] / 2) inb = false;
        if (!inb) continue;
        // global_interp's stencil (fmisc.f90:738-781)
        const std::vector<double>* co[3] = {&b.X, &b.Y, &b.Z};
        InterpItem t;
        for (int d = 0; d < 3; ++d) {
          const std::vector<double>& c = *co[d];
          const double dd = c[1] - c[0];
          const int cxI = (int)((pt[d] - c[0]) / dd + 0.4) + 1;
          int cxB = cxI - 2, cxT = cxB + 5;
          const bool mirror = (d < 2 && e->prm.symmetry == 2) || (d == 2 && e->prm.symmetry != 0);
          const int cmin = mirror && std::fabs(c[0]) < dd ? -2 : 1;
          if (cxB < cmin) { cxB = cmin; cxT = cxB + 5; }
          if (cxT > b.ex[d]) { cxT = b.ex[d]; cxB = cxT - 5; }
          if (cxT > b.ex[d] || (cxB <= 0 && 1 - cxB > b.ex[d]))
            return amss_fail(AMSS_ERR_ARG, "amss_engine_interp_points: stencil outside the block (decide3d)");
          t.ex[d] = b.ex[d];
          t.cxB[d] = cxB;
          t.cx[d] = cxB > 0 ? (pt[d] - c[cxB - 1]) / dd : (pt[d] + c[-cxB]) / dd;
        }
        const double* u = from_acc ? b.K : cur_state(e, b);
        for (int v = 0; v < nvar; ++v) {
          t.f = u + (long long)fields[v] * b.fs;
          for (int d = 0; d < 3; ++d) t.soa[d] = soa ? soa[3 * v + d] : 1.0;
          items.push_back(t);
          where.push_back((long long)p * nvar + v);
        }
        ok = 1;
        break;
      }
      if (!ok) return amss_fail(AMSS_ERR_ARG, "amss_engine_interp_points: a point of a patch lies in none of its blocks");
      break;
    }
    if (found) found[p] = ok;
    if (!ok)
      for (int v = 0; v < nvar; ++v) out[(long long)p * nvar + v] = 0.0;
  }
  const long long n = (long long)items.size();
  if (n == 0) return 0;
  if (e->icap < n) {
    if (e->iitems) cudaFree(e->iitems);
    if (e->iout) cudaFree(e->iout);
    e->iitems = nullptr;
    e->iout = nullptr;
    e->icap = 0;
    AMSS_CK(cudaMalloc(&e->iitems, n * sizeof(InterpItem)));
    AMSS_CK(cudaMalloc(&e->iout, n * sizeof(double)));
    e->icap = n;
  }
  AMSS_CK(cudaMemcpyAsync(e->iitems, items.data(), n * sizeof(InterpItem), cudaMemcpyHostToDevice, e->stream));
  AMSS_CK(launch_interp_points(e->iitems, (int)n, e->iout, e->stream));
  e->launches++;
  std::vector<double> res(n);
  AMSS_CK(cudaMemcpyAsync(res.data(), e->iout, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  for (long long i = 0; i < n; ++i) out[where[i]] = res[i];
  return 0;
}

extern "C" int amss_engine_interp_points(amss_engine* e, int level, int npts, const double* xyz, int nvar,
                                         const int* fields, const double* soa, double* out, int* found) {
  return interp_level(e, level, npts, xyz, nvar, fields, soa, out, found, false);
}

// bssn_class::Compute_Psi4 (bssn_class.C:6210-6298): Psi4 of the level's
// current state on every point of its blocks, then the level's ghost sync.
extern "C" int amss_engine_psi4(amss_engine* e, int level) {
  if (!e || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "amss_engine_psi4: commit the engine first");
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_psi4: no such level");
  ELevel& L = it->second;
  if (!L.own.empty()) {
    if (e->pscr_cap < 24 * L.dfs) {
      if (e->pscr) cudaFree(e->pscr);
      e->pscr = nullptr;
      e->pscr_cap = 0;
      AMSS_CK(cudaMalloc(&e->pscr, (size_t)24 * L.dfs * sizeof(double)));
      e->pscr_cap = 24 * L.dfs;
    }
    const int tile_pts = e->prm.kernel == 0 ? (int)kPointwiseTile : 128;
    const cudaError_t err =
        e->prm.precision == 1
            ? launch_psi4<float>(L.dtable, L.dtiles, L.ntiles, tile_pts, L.symm, e->pscr, L.dfs, e->stream)
            : launch_psi4<double>(L.dtable, L.dtiles, L.ntiles, tile_pts, L.symm, e->pscr, L.dfs, e->stream);
    AMSS_CK(err);
    e->launches += 2;
  }
  return run_xfer(e, L.xsync, BUF_TEMP);   // Parallel::Sync of Rpsi4 / Ipsi4
}

extern "C" int amss_engine_get_psi4(amss_engine* e, int block, double* h) {
  if (int rc = check_block(e, block)) return rc;
  if (!h) return amss_fail(AMSS_ERR_ARG, "amss_engine_get_psi4: null buffer");
  EBlock& b = e->blocks[block];
  AMSS_CK(cudaMemcpy2DAsync(h, b.npts * sizeof(double), b.K, b.fs * sizeof(double), b.npts * sizeof(double), 2,
                            cudaMemcpyDeviceToHost, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  return 0;
}

// The sphere of surface_integral::surface_integral (surface_integral.C:39-181,
// GaussInt): N_theta = 2N Gauss-Legendre nodes in cos(theta), upper
// hemisphere first, N_phi = 4N midpoints in phi; Symmetry 1 keeps the upper
// half, Symmetry 2 also a quarter in phi (factor: the copies it stands for).
struct Sphere {
  int n_theta, n_phi, ntot, factor;
  double dphi;
  std::vector<double> ct, wt, nx, ny, nz, xyz;
};
static Sphere make_sphere(int nquarter, int sym, double rex) {
  Sphere S;
  S.n_phi = 4 * nquarter;
  S.n_theta = 2 * nquarter;
  gauss_legendre_desc(S.n_theta, S.ct, S.wt);
  if (sym == 2) {
    S.n_phi /= 4;
    S.n_theta /= 2;
    S.dphi = M_PI / (2.0 * S.n_phi);
    S.factor = 8;
  } else if (sym == 1) {
    S.n_theta /= 2;
    S.dphi = 2.0 * M_PI / S.n_phi;
    S.factor = 2;
  } else {
    S.dphi = 2.0 * M_PI / S.n_phi;
    S.factor = 1;
  }
  S.ntot = S.n_theta * S.n_phi;
  S.xyz.resize(3 * (size_t)S.ntot);
  S.nx.resize(S.ntot);
  S.ny.resize(S.ntot);
  S.nz.resize(S.ntot);
  for (int i = 0, n = 0; i < S.n_theta; ++i) {
    const double s = std::sqrt(1.0 - S.ct[i] * S.ct[i]);
    for (int j = 0; j < S.n_phi; ++j, ++n) {
      const double ph = (j + 0.5) * S.dphi;
      S.nx[n] = s * std::cos(ph);
      S.ny[n] = s * std::sin(ph);
      S.nz[n] = S.ct[i];
      S.xyz[3 * n] = rex * S.nx[n];
      S.xyz[3 * n + 1] = rex * S.ny[n];
      S.xyz[3 * n + 2] = rex * S.nz[n];
    }
  }
  return S;
}

// surface_integral::surf_Wave (surface_integral.C:197-377, GaussInt; sphere of
// surface_integral.C:39-181): Psi4 of the level (amss_engine_psi4 first)
// interpolated at N_theta x N_phi points of the sphere of radius rex --
// Gauss-Legendre nodes in cos(theta) (the upper hemisphere first), midpoints
// in phi, N_theta = 2N, N_phi = 4N, halved in theta for Symmetry 1 and also
// quartered in phi for Symmetry 2 -- and projected on the spin-weight -2
// harmonics, l = 2..maxl, m = -l..l; the mirrored parts of the sphere enter
// through the parities of Rpsi4 (+, +, +) and Ipsi4 (-, -, -).
extern "C" int amss_engine_psi4_modes(amss_engine* e, int level, double rex, int nquarter, int maxl, double* RP,
                                      double* IP) {
  if (!RP || !IP || !(rex > 0) || nquarter < 1 || maxl < 2)
    return amss_fail(AMSS_ERR_ARG, "amss_engine_psi4_modes: rex > 0, N >= 1, maxl >= 2 and output arrays");
  if (int rc = check_whole(e, "amss_engine_psi4_modes")) return rc;
  const int sym = e->prm.symmetry;
  const Sphere S = make_sphere(nquarter, sym, rex);
  const int n_phi = S.n_phi, ntot = S.ntot;
  const double dphi = S.dphi;
  const std::vector<double>& ct = S.ct;
  const std::vector<double>& wt = S.wt;
  const std::vector<double>& xyz = S.xyz;
  const int fields[2] = {0, 1};
  const double soa[6] = {1, 1, 1, -1, -1, -1};   // Rpsi4, Ipsi4 (bssn_class.C:347-348)
  std::vector<double> v(2 * (size_t)ntot);
  std::vector<int> found(ntot);
  if (int rc = interp_level(e, level, ntot, xyz.data(), 2, fields, soa, v.data(), found.data(), true)) return rc;
  for (int n = 0; n < ntot; ++n)
    if (!found[n]) return amss_fail(AMSS_ERR_ARG, "amss_engine_psi4_modes: the sphere leaves the level's patches");
  const int nn = (maxl + 1) * (maxl + 1) - 4;
  std::vector<double> rp(nn, 0.0), ip(nn, 0.0);
  const int lpsy = sym == 0 ? 1 : (sym == 1 ? 2 : 8);
  // per mirror image lp: the sign of cos(theta), the phi map, the parity factors
  for (int n = 0; n < ntot; ++n) {
    const int i = n / n_phi, j = n - i * n_phi;
    const double R = v[2 * n], I = v[2 * n + 1];
    int c = 0;
    for (int l = 2; l <= maxl; ++l)
      for (int m = -l; m <= l; ++m, ++c)
        for (int lp = 0; lp < lpsy; ++lp) {
          const bool flip_z = lp & 1, flip_y = (lp == 2 || lp == 3 || lp == 6 || lp == 7), flip_x = lp >= 4;
          const double cth = flip_z ? -ct[i] : ct[i];
          double arg;
          if (lp < 4) arg = m * (j + 0.5) * dphi;
          else if (lp < 6) arg = m * (M_PI - (j + 0.5) * dphi);
          else arg = m * (M_PI + (j + 0.5) * dphi);
          const double cm = std::cos(arg);
          const double sm = (lp == 2 || lp == 3) ? -std::sin(arg) : std::sin(arg);
          // Rpsi4 is even in every direction; Ipsi4 odd in each flipped one
          const double sI = ((flip_x ? -1.0 : 1.0) * (flip_y ? -1.0 : 1.0)) * (flip_z ? -1.0 : 1.0);
          const double r = R, im = sI * I;
          const double th = std::sqrt((2 * l + 1.0) / 4.0 / M_PI) * wigner_d(l, m, 2, cth);
          rp[c] = rp[c] + th * (r * cm + im * sm) * wt[i];
          ip[c] = ip[c] + th * (im * cm - r * sm) * wt[i];
        }
  }
  for (int c = 0; c < nn; ++c) {
    RP[c] = rp[c] * rex * dphi;
    IP[c] = ip[c] * rex * dphi;
  }
  return 0;
}

// surface_integral::surf_MassPAng (surface_integral.C:2247-2512, GaussInt):
// the ADM mass, linear and angular momentum through the sphere of radius rex
// on a level.  The mass integrand of admmass_bssn is formed on the level's
// blocks (accumulator fields 2-4, not synchronised, as the reference leaves
// its temporaries), interpolated with chi, trK, the metric and A~ij at the
// sphere's points, and summed with the Gauss-Legendre weights.  Symmetry 1
// integrates S_z, P_x and P_y only, Symmetry 2 the mass only (the others 0).
// out: mass, Px, Py, Pz, Sx, Sy, Sz (the bssn_ADMQs.dat columns).
extern "C" int amss_engine_adm_integrals(amss_engine* e, int level, double rex, int nquarter, double* out) {
  if (!out || !(rex > 0) || nquarter < 1)
    return amss_fail(AMSS_ERR_ARG, "amss_engine_adm_integrals: rex > 0, N >= 1 and an output array");
  if (int rc = check_whole(e, "amss_engine_adm_integrals")) return rc;
  auto it = e->levels.find(level);
  if (it == e->levels.end()) return amss_fail(AMSS_ERR_ARG, "amss_engine_adm_integrals: no such level");
  ELevel& L = it->second;
  const int tile_pts = e->prm.kernel == 0 ? (int)kPointwiseTile : 128;
  AMSS_CK(e->prm.precision == 1 ? launch_admmass<float>(L.dtable, L.dtiles, L.ntiles, tile_pts, L.symm, e->stream)
                                : launch_admmass<double>(L.dtable, L.dtiles, L.ntiles, tile_pts, L.symm, e->stream));
  e->launches++;
  const int sym = e->prm.symmetry;
  const Sphere S = make_sphere(nquarter, sym, rex);
  const int ntot = S.ntot;
  // the mass integrand has the shift's parities; chi .. A~zz the state's
  const int mfields[3] = {2, 3, 4};
  const double msoa[9] = {-1, 1, 1, 1, -1, 1, 1, 1, -1};
  const int sfields[14] = {F_CHI, F_TRK, F_GXX, F_GXY, F_GXZ, F_GYY, F_GYZ, F_GZZ,
                           F_AXX, F_AXY, F_AXZ, F_AYY, F_AYZ, F_AZZ};
  double ssoa[42];
  for (int v = 0; v < 14; ++v)
    for (int d = 0; d < 3; ++d) ssoa[3 * v + d] = soa_sign(sfields[v], d);
  std::vector<double> mv(3 * (size_t)ntot), sv(14 * (size_t)ntot);
  std::vector<int> found(ntot);
  if (int rc = interp_level(e, level, ntot, S.xyz.data(), 3, mfields, msoa, mv.data(), found.data(), true)) return rc;
  for (int n = 0; n < ntot; ++n)
    if (!found[n]) return amss_fail(AMSS_ERR_ARG, "amss_engine_adm_integrals: the sphere leaves the level's patches");
  if (int rc = interp_level(e, level, ntot, S.xyz.data(), 14, sfields, ssoa, sv.data(), nullptr, false)) return rc;
  const double f1o8 = 0.125;
  double mass = 0, sx = 0, sy = 0, sz = 0, px = 0, py = 0, pz = 0;
  for (int n = 0; n < ntot; ++n) {
    const int i = n / S.n_phi;
    const double* m = &mv[3 * (size_t)n];
    const double* s = &sv[14 * (size_t)n];
    const double nx = S.nx[n], ny = S.ny[n], nz = S.nz[n], w = S.wt[i];
    const double X = S.xyz[3 * n], Y = S.xyz[3 * n + 1], Z = S.xyz[3 * n + 2];
    double Chi = s[0];
    const double TRK = s[1];
    const double Gxx = s[2] + 1.0, Gxy = s[3], Gxz = s[4], Gyy = s[5] + 1.0, Gyz = s[6], Gzz = s[7] + 1.0;
    double axx = s[8], axy = s[9], axz = s[10], ayy = s[11], ayz = s[12], azz = s[13];
    Chi = 1.0 / (1.0 + Chi);          // psi^4
    const double Psi = Chi * std::sqrt(Chi);   // psi^6
    mass = mass + (m[0] * nx + m[1] * ny + m[2] * nz) * w;
    double gupzz = Gxx * Gyy * Gzz + Gxy * Gyz * Gxz + Gxz * Gxy * Gyz - Gxz * Gyy * Gxz - Gxy * Gxy * Gzz -
                   Gxx * Gyz * Gyz;
    const double gupxx = (Gyy * Gzz - Gyz * Gyz) / gupzz;
    const double gupxy = -(Gxy * Gzz - Gyz * Gxz) / gupzz;
    const double gupxz = (Gxy * Gyz - Gyy * Gxz) / gupzz;
    const double gupyy = (Gxx * Gzz - Gxz * Gxz) / gupzz;
    const double gupyz = -(Gxx * Gyz - Gxy * Gxz) / gupzz;
    gupzz = (Gxx * Gyy - Gxy * Gxy) / gupzz;
    const double aupxx = gupxx * axx + gupxy * axy + gupxz * axz;
    const double aupxy = gupxx * axy + gupxy * ayy + gupxz * ayz;
    const double aupxz = gupxx * axz + gupxy * ayz + gupxz * azz;
    const double aupyx = gupxy * axx + gupyy * axy + gupyz * axz;
    const double aupyy = gupxy * axy + gupyy * ayy + gupyz * ayz;
    const double aupyz = gupxy * axz + gupyy * ayz + gupyz * azz;
    const double aupzx = gupxz * axx + gupyz * axy + gupzz * axz;
    const double aupzy = gupxz * axy + gupyz * ayy + gupzz * ayz;
    const double aupzz = gupxz * axz + gupyz * ayz + gupzz * azz;
    // 1/8pi \int psi^6 (x^a A^m_b - x^b A^m_a) dS_m
    if (sym == 0) {
      sx = sx + f1o8 * Psi * (nx * (Y * aupxz - Z * aupxy) + ny * (Y * aupyz - Z * aupyy) + nz * (Y * aupzz - Z * aupzy)) * w;
      sy = sy + f1o8 * Psi * (nx * (Z * aupxx - X * aupxz) + ny * (Z * aupyx - X * aupyz) + nz * (Z * aupzx - X * aupzz)) * w;
    }
    if (sym == 0 || sym == 1)
      sz = sz + f1o8 * Psi * (nx * (X * aupxy - Y * aupxx) + ny * (X * aupyy - Y * aupyx) + nz * (X * aupzy - Y * aupzx)) * w;
    axx = Chi * (axx + Gxx * TRK / 3.0);
    axy = Chi * (axy + Gxy * TRK / 3.0);
    axz = Chi * (axz + Gxz * TRK / 3.0);
    ayy = Chi * (ayy + Gyy * TRK / 3.0);
    ayz = Chi * (ayz + Gyz * TRK / 3.0);
    azz = Chi * (azz + Gzz * TRK / 3.0);
    axx = axx - TRK;
    ayy = ayy - TRK;
    azz = azz - TRK;
    // 1/8pi \int psi^6 (K_mi - delta_mi K) dS^m
    if (sym == 0 || sym == 1) {
      px = px + f1o8 * Psi * (nx * axx + ny * axy + nz * axz) * w;
      py = py + f1o8 * Psi * (nx * axy + ny * ayy + nz * ayz) * w;
    }
    if (sym == 0) pz = pz + f1o8 * Psi * (nx * axz + ny * ayz + nz * azz) * w;
  }
  out[0] = mass * rex * rex * S.dphi * S.factor;
  out[1] = px * rex * rex * S.dphi * (1.0 / M_PI) * S.factor;
  out[2] = py * rex * rex * S.dphi * (1.0 / M_PI) * S.factor;
  out[3] = pz * rex * rex * S.dphi * (1.0 / M_PI) * S.factor;
  out[4] = sx * rex * rex * S.dphi * (1.0 / M_PI) * S.factor;
  out[5] = sy * rex * rex * S.dphi * (1.0 / M_PI) * S.factor;
  out[6] = sz * rex * rex * S.dphi * (1.0 / M_PI) * S.factor;
  return 0;
}

// Puncture tracking (bssn_class::Step with MAPBH 0, bssn_class.C:3360-3390,
// :3730-3760, :3804-3812, :3890-3898): positions advanced by RK4 with the
// finest level's substeps, on the device inside the step (and its graphs).
extern "C" int amss_engine_set_punctures(amss_engine* e, int n, const double* pos) {
  if (!e || n < 0 || n > kMaxPunctures || (n > 0 && !pos))
    return amss_fail(AMSS_ERR_ARG, "amss_engine_set_punctures: 0 <= n <= 10 positions");
  if (!e->committed) return amss_fail(AMSS_ERR_STATE, "amss_engine_set_punctures: commit the engine first");
  if (int rc = check_whole(e, "amss_engine_set_punctures")) return rc;
  e->ntrack = 0;
  if (n == 0) return 0;
  const int level = e->levels.rbegin()->first;
  // the reference drops the buffer on a patch side moved onto a symmetry plane
  // (MPatch.C:79-116); the engine's patches carry one buffer width on every side
  if (e->prm.symmetry > 0)
    for (int pid : e->levels[level].patches)
      if (e->patches[pid].buffer > 0)
        return amss_fail(AMSS_ERR_UNSUPPORTED, "amss_engine_set_punctures: symmetry planes with buffered refined "
                                               "patches on the finest level are not supported");
  const std::vector<IPatch> ps = level_patches(e, e->levels[level]);
  std::vector<TrackPatch> tp;
  std::vector<TrackBlock> tb;
  for (const auto& q : ps) {
    TrackPatch P;
    for (int d = 0; d < 3; ++d) {
      P.lo[d] = q.pbb[d] + q.buffer * q.h[d];
      P.hi[d] = q.pbb[3 + d] - q.buffer * q.h[d];
      P.half[d] = q.h[d] / 2;
    }
    P.b0 = (int)tb.size();
    for (int bid : q.blocks) {
      const EBlock& b = e->blocks[bid];
      TrackBlock B;
      for (int t = 0; t < 3; ++t) B.tl[t] = b.tl[t];
      B.stage[0] = b.st[0];
      B.stage[1] = b.st[1];
      B.side[0] = b.side[0];
      B.side[1] = b.side[1];
      B.f32 = e->prm.precision == 1;
      B.fs = b.fs;
      find_box(b, q, B.flo, B.fhi);
      const std::vector<double>* co[3] = {&b.X, &b.Y, &b.Z};
      for (int d = 0; d < 3; ++d) {
        B.ex[d] = b.ex[d];
        B.blo[d] = b.bbox[d];
        B.bh[d] = (b.bbox[3 + d] - b.bbox[d]) / b.ex[d];
        B.x0[d] = (*co[d])[0];
        B.dd[d] = (*co[d])[1] - (*co[d])[0];
        const bool mirror = (d < 2 && e->prm.symmetry == 2) || (d == 2 && e->prm.symmetry != 0);
        B.cmin[d] = mirror && std::fabs(B.x0[d]) < B.dd[d] ? -2 : 1;
      }
      tb.push_back(B);
    }
    P.b1 = (int)tb.size();
    tp.push_back(P);
  }
  if (e->dtpatch) cudaFree(e->dtpatch);
  if (e->dtblock) cudaFree(e->dtblock);
  e->dtpatch = nullptr;
  e->dtblock = nullptr;
  AMSS_CK(cudaMalloc(&e->dtpatch, tp.size() * sizeof(TrackPatch)));
  AMSS_CK(cudaMalloc(&e->dtblock, tb.size() * sizeof(TrackBlock)));
  if (!e->dtrack) AMSS_CK(cudaMalloc(&e->dtrack, sizeof(TrackState)));
  TrackState S;
  std::memset(&S, 0, sizeof S);
  for (int i = 0; i < 3 * n; ++i) {
    if (!std::isfinite(pos[i])) return amss_fail(AMSS_ERR_ARG, "amss_engine_set_punctures: a position is not finite");
    S.p0[i] = pos[i];
  }
  AMSS_CK(cudaMemcpyAsync(e->dtpatch, tp.data(), tp.size() * sizeof(TrackPatch), cudaMemcpyHostToDevice, e->stream));
  AMSS_CK(cudaMemcpyAsync(e->dtblock, tb.data(), tb.size() * sizeof(TrackBlock), cudaMemcpyHostToDevice, e->stream));
  AMSS_CK(cudaMemcpyAsync(e->dtrack, &S, sizeof S, cudaMemcpyHostToDevice, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  e->ntpatch = (int)tp.size();
  e->track_level = level;
  e->ntrack = n;
  return 0;
}

extern "C" int amss_engine_get_punctures(amss_engine* e, double* pos) {
  if (!e || !pos) return amss_fail(AMSS_ERR_ARG, "amss_engine_get_punctures: null argument");
  if (e->ntrack == 0) return amss_fail(AMSS_ERR_STATE, "amss_engine_get_punctures: no punctures set");
  TrackState S;
  AMSS_CK(cudaMemcpyAsync(&S, e->dtrack, sizeof S, cudaMemcpyDeviceToHost, e->stream));
  AMSS_CK(cudaStreamSynchronize(e->stream));
  for (int i = 0; i < 3 * e->ntrack; ++i) pos[i] = S.p0[i];
  if (S.err) return amss_fail(AMSS_ERR_STATE, "amss_engine_get_punctures: a puncture left the finest level");
  return 0;
}
