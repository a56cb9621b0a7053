// xfer.cu -- the data movements between blocks (same-level ghost sync,
// restriction into the parent level, prolongation into the buffer cells) as
// box lists, divided among the ranks that own the blocks, and their exchange
// between ranks.
//
// The reference moves the same boxes with MPI: Parallel::transfer
// (Parallel.C:3508-3592) packs every segment whose source it holds -- the
// restriction and prolongation are applied while packing -- sends it to the
// rank that holds the destination and unpacks what it receives.  Here the
// packing is the transfer's own kernel writing into staging blocks (extra
// entries of the AMR block table whose arrays are regions of a staging arena),
// the exchange moves whole per-peer regions of that arena, and the unpacking is
// the ghost-sync kernel reading the received staging blocks.  Two transports:
//   * in-process ranks (amss_group): one engine per GPU in one process, driven
//     by one host thread each; every rank records an event after its packing,
//     the ranks meet at a host barrier (with a timeout), each pulls its
//     regions from the peers' staging arenas with device-to-device copies
//     ordered after the peers' events, and a second barrier plus event waits
//     keep a peer's arena from being refilled before it has been read;
//   * NCCL: grouped ncclSend / ncclRecv of the same regions on the engine's
//     stream (libnccl is opened at run time; its handle, unique id and rank
//     layout come from the caller).
// No kernel of one rank waits on another rank's kernel: the ordering is
// stream order, events and host barriers.
#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <nccl.h>

#include "engine_internal.cuh"

struct amss_group {
  int n = 0;
  std::vector<amss_engine*> eng;   // by rank
  std::mutex mu;
  std::condition_variable cv;
  int arrived = 0;
  long long gen = 0;
  bool broken = false;
  double timeout_s = 60.0;
};

namespace amss {

cudaError_t launch_amr_sync(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles, int which,
                            bool fp32_stages, unsigned* status, cudaStream_t s);
cudaError_t launch_amr_prolong(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles,
                               int from_temp, unsigned* status, cudaStream_t s);
cudaError_t launch_amr_restrict(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles,
                                int to_temp, unsigned* status, cudaStream_t s);

// Same-level ghost fill (Parallel::Sync, Parallel.C:3677-3776): every cell of a
// block's array that another block of the level owns is copied from it.
static std::vector<AmrBox> sync_boxes(amss_engine* e, const ELevel& L) {
  std::vector<AmrBox> v;
  for (int d : L.blocks)
    for (int s : L.blocks)
      if (d != s) push_box(v, d, s, intersect(e->blocks[d].array(), e->blocks[s].own));
  return v;
}

// Restriction (Parallel::Restrict, Parallel.C:4485-4543): every cell of a
// parent block's array (ghosts included) inside a child patch's physical
// region, from the child block that owns its two children per direction.
static std::vector<AmrBox> restrict_boxes(amss_engine* e, const ELevel& F, const ELevel& C) {
  std::vector<AmrBox> v;
  for (int pid : F.patches) {
    const EPatch& P = e->patches[pid];
    Box cphys;
    for (int d = 0; d < 3; ++d) { cphys.lo[d] = P.phys.lo[d] / 2; cphys.hi[d] = P.phys.hi[d] / 2; }
    for (int cb : C.blocks) {
      const Box r = intersect(cphys, e->blocks[cb].array());
      if (r.empty()) continue;
      for (int fb : P.blocks) {
        const Box& o = e->blocks[fb].own;
        Box oc;
        for (int d = 0; d < 3; ++d) { oc.lo[d] = o.lo[d] / 2; oc.hi[d] = o.hi[d] / 2; }
        push_box(v, cb, fb, intersect(r, oc));
      }
    }
  }
  return v;
}

// Prolongation into the buffer cells (Parallel::OutBdLow2Hi,
// Parallel.C:4589-4689): every cell of a child block's array in its patch's
// buffer region, from the parent block that owns the cell's parent.
static std::vector<AmrBox> prolong_boxes(amss_engine* e, const ELevel& F, const ELevel& C) {
  std::vector<AmrBox> v;
  for (int pid : F.patches) {
    const EPatch& P = e->patches[pid];
    const Box ext = P.ext();
    std::vector<Box> slabs;
    for (int d = 0; d < 3; ++d) {
      Box lo = ext, hi = ext;
      for (int q = 0; q < d; ++q) { lo.lo[q] = hi.lo[q] = P.phys.lo[q]; lo.hi[q] = hi.hi[q] = P.phys.hi[q]; }
      lo.hi[d] = P.phys.lo[d];
      hi.lo[d] = P.phys.hi[d];
      slabs.push_back(lo);
      slabs.push_back(hi);
    }
    for (int fb : P.blocks)
      for (const Box& s : slabs) {
        const Box r = intersect(s, e->blocks[fb].array());
        if (r.empty()) continue;
        for (int cb : C.blocks) {
          const Box& o = e->blocks[cb].own;
          Box of;
          for (int d = 0; d < 3; ++d) { of.lo[d] = 2 * o.lo[d]; of.hi[d] = 2 * o.hi[d]; }
          push_box(v, fb, cb, intersect(r, of));
        }
      }
  }
  return v;
}

// ---- plans ------------------------------------------------------------------

static long long align256(long long x) { return (x + 255) / 256 * 256; }

// Bytes of the staging block of a box: the nf FP64 fields of the state or the
// accumulator, or the stage fields (FP32 in the mixed form, then its FP64 side
// fields) -- whichever buffer the transfer moves; all of them start at the
// block's base.
static long long stage_bytes(const amss_engine* e, const AmrBox& b) {
  const long long n = (long long)b.n[0] * b.n[1] * b.n[2];
  const bool mixed = e->prm.precision == 1;
  const long long full = align256((long long)e->nf * n * 8);
  const long long stage = align256((long long)e->nf * n * (mixed ? 4 : 8)) + (mixed ? align256((long long)kSideFields * n * 8) : 0);
  return std::max(full, stage);
}

static int add_stage(amss_engine* e, const AmrBox& b, long long off, int in) {
  XStage s;
  for (int d = 0; d < 3; ++d) { s.org[d] = b.lo[d]; s.ex[d] = b.n[d]; }
  s.off = off;
  s.in = in;
  e->staging.push_back(s);
  return (int)e->blocks.size() + (int)e->staging.size() - 1;
}

// This rank's share of a transfer whose full box list is `all`.  The staging
// regions are laid out per peer in rank order and, within a peer, in the
// order of the full list, so sender and receiver agree without talking.
static int plan_xfer(amss_engine* e, int kind, int level, const std::vector<AmrBox>& all) {
  XferOp op;
  op.kind = kind;
  op.level = level;
  op.nall = (long long)all.size();
  const int me = e->rank;
  for (const AmrBox& b : all) {
    const int od = e->blocks[b.dst].owner, os = e->blocks[b.src].owner;
    if (od != os) op.ncross++;
    if (od == me && os == me) op.run_h.push_back(b);
  }
  for (int q = 0; q < e->nranks; ++q) {
    if (q == me) continue;
    XPeer s{q, op.out_bytes, 0};
    for (const AmrBox& b : all) {
      if (e->blocks[b.src].owner != me || e->blocks[b.dst].owner != q) continue;
      AmrBox r = b;
      r.dst = add_stage(e, b, op.out_bytes, 0);
      op.run_h.push_back(r);
      op.out_bytes += stage_bytes(e, b);
    }
    s.bytes = op.out_bytes - s.off;
    if (s.bytes) op.send.push_back(s);
    XPeer r{q, op.in_bytes, 0};
    for (const AmrBox& b : all) {
      if (e->blocks[b.dst].owner != me || e->blocks[b.src].owner != q) continue;
      AmrBox u = b;
      u.src = add_stage(e, b, op.in_bytes, 1);
      op.unpack_h.push_back(u);
      op.in_bytes += stage_bytes(e, b);
    }
    r.bytes = op.in_bytes - r.off;
    if (r.bytes) op.recv.push_back(r);
  }
  e->xfers.push_back(std::move(op));
  return (int)e->xfers.size() - 1;
}

// ---- final-substep regions ---------------------------------------------------
// In a coarse step every level step of a refined level is followed by its
// RestrictProlong (bssn_class.C:5724-5903): the restriction reads the level's
// new state around its physical boxes, then the prolongation overwrites the
// level's buffer cells.  In between, only the finer levels' prolongation reads
// the level (its new state, or the time interpolation formed from it).  Where
// each of these reads, and every physical cell, stays within kFinalPad cells
// of the physical box of the block that owns the cell, and the prolongation
// covers every buffer cell of the level's arrays, the final RK4 substep need
// not update the owned cells further out: nothing reads their new values
// before the prolongation replaces them.  The state after the coarse step is
// the same bit for bit.
static const int kFinalPad = 2;   // restrict3 reads fine cells 2k-2 .. 2k+3

static Box grow(const Box& b, int g) {
  Box r = b;
  for (int d = 0; d < 3; ++d) { r.lo[d] -= g; r.hi[d] += g; }
  return r;
}
static long long volume(const Box& b) {
  return b.empty() ? 0 : (long long)(b.hi[0] - b.lo[0]) * (b.hi[1] - b.lo[1]) * (b.hi[2] - b.lo[2]);
}

// Every cell of R is owned by a block of L within pad of its patch's physical box.
static bool reads_valid(const amss_engine* e, const ELevel& L, const Box& R, int pad) {
  long long cov = 0;
  for (int y : L.blocks) {
    const EBlock& Y = e->blocks[y];
    const Box s = intersect(R, Y.own);
    if (s.empty()) continue;
    const Box ok = intersect(s, grow(e->patches[Y.patch].phys, pad));
    if (volume(ok) != volume(s)) return false;
    cov += volume(s);
  }
  return cov == volume(R);
}

Box final_region(const amss_engine* e, const ELevel& L, const EBlock& b) {
  if (L.final_pad < 0 || b.patch < 0) return b.array();
  return intersect(intersect(b.own, grow(e->patches[b.patch].phys, L.final_pad)), b.array());
}

void plan_final_regions(amss_engine* e) {
  for (auto& kv : e->levels) {
    kv.second.final_pad = -1;
    kv.second.own_ok = false;
  }
  // owned cells only: owned boxes disjoint and inside the arrays, and the
  // sync's boxes into each block cover every cell of its array it does not own
  for (auto& kv : e->levels) {
    ELevel& L = kv.second;
    bool ok = !L.blocks.empty();
    std::map<int, long long> cover;
    for (const AmrBox& b : sync_boxes(e, L)) cover[b.dst] += (long long)b.n[0] * b.n[1] * b.n[2];
    for (size_t a = 0; a < L.blocks.size() && ok; ++a) {
      const EBlock& A = e->blocks[L.blocks[a]];
      if (volume(intersect(A.own, A.array())) != volume(A.own) || volume(A.own) == 0) ok = false;
      if (cover[L.blocks[a]] != volume(A.array()) - volume(A.own)) ok = false;
      for (size_t b = a + 1; b < L.blocks.size() && ok; ++b)
        if (volume(intersect(A.own, e->blocks[L.blocks[b]].own)) != 0) ok = false;
    }
    L.own_ok = ok;
  }
  for (auto& kv : e->levels) {
    const int l = kv.first;
    ELevel& L = kv.second;
    if (l == 0 || L.blocks.empty() || !e->levels.count(l - 1)) continue;
    const ELevel& C = e->levels.at(l - 1);
    bool ok = true;
    // blocks of buffered patches, owned boxes disjoint
    for (size_t a = 0; a < L.blocks.size() && ok; ++a) {
      const EBlock& A = e->blocks[L.blocks[a]];
      if (A.patch < 0 || e->patches[A.patch].buffer <= 0) ok = false;
      for (size_t b = a + 1; b < L.blocks.size() && ok; ++b)
        if (volume(intersect(A.own, e->blocks[L.blocks[b]].own)) != 0) ok = false;
    }
    if (!ok) continue;
    // the prolongation into the level writes every array cell outside the
    // physical box; the physical cells are valid
    std::map<int, long long> cover;
    for (const AmrBox& b : prolong_boxes(e, L, C)) cover[b.dst] += (long long)b.n[0] * b.n[1] * b.n[2];
    for (int x : L.blocks) {
      const EBlock& X = e->blocks[x];
      const Box ph = intersect(X.array(), e->patches[X.patch].phys);
      if (cover[x] != volume(X.array()) - volume(ph) || !reads_valid(e, L, ph, kFinalPad)) { ok = false; break; }
    }
    // the restriction out of the level: fine 2k-2 .. 2k+3 of coarse cell k
    if (ok)
      for (const AmrBox& b : restrict_boxes(e, L, C)) {
        Box R;
        for (int d = 0; d < 3; ++d) { R.lo[d] = 2 * b.lo[d] - 2; R.hi[d] = 2 * (b.lo[d] + b.n[d]) + 2; }
        if (!reads_valid(e, L, R, kFinalPad)) { ok = false; break; }
      }
    // the prolongation into the next finer level: coarse (g >> 1) - 3 .. + 2 of
    // an even fine cell g, (g >> 1) - 2 .. + 3 of an odd one
    if (ok && e->levels.count(l + 1))
      for (const AmrBox& b : prolong_boxes(e, e->levels.at(l + 1), L)) {
        Box R;
        for (int d = 0; d < 3; ++d) {
          const int g0 = b.lo[d], g1 = b.lo[d] + b.n[d] - 1;
          R.lo[d] = (g0 & 1) ? (g0 >> 1) - 2 : (g0 >> 1) - 3;
          R.hi[d] = ((g1 & 1) ? (g1 >> 1) - 2 : (g1 >> 1) - 3) + 6;
        }
        if (!reads_valid(e, L, R, kFinalPad)) { ok = false; break; }
      }
    if (ok) L.final_pad = kFinalPad;
  }
}

// The cells of each of this rank's blocks of C (level l-1) whose time
// interpolation the prolongation into F (level l) reads: per block the
// bounding box of its owned cells inside the prolongation's coarse read boxes
// (prolong3: coarse (g >> 1) - 3 .. + 2 of an even fine cell g, (g >> 1) - 2
// .. + 3 of an odd one).  A read box's ghost cells are owned by another block
// of C, whose own box covers them and whose values the temp sync copies.
std::vector<AmrBox> timeinterp_boxes(amss_engine* e, const ELevel& C, const ELevel& F) {
  std::vector<Box> reads;
  for (const AmrBox& b : prolong_boxes(e, F, C)) {
    Box R;
    for (int d = 0; d < 3; ++d) {
      const int g0 = b.lo[d], g1 = b.lo[d] + b.n[d] - 1;
      R.lo[d] = (g0 & 1) ? (g0 >> 1) - 2 : (g0 >> 1) - 3;
      R.hi[d] = ((g1 & 1) ? (g1 >> 1) - 2 : (g1 >> 1) - 3) + 6;
    }
    reads.push_back(R);
  }
  std::vector<AmrBox> v;
  for (int x : C.own) {
    const EBlock& X = e->blocks[x];
    Box h{{0, 0, 0}, {0, 0, 0}};
    bool any = false;
    for (const Box& R : reads) {
      const Box s = intersect(R, X.own);
      if (s.empty()) continue;
      for (int d = 0; d < 3; ++d) {
        h.lo[d] = any ? std::min(h.lo[d], s.lo[d]) : s.lo[d];
        h.hi[d] = any ? std::max(h.hi[d], s.hi[d]) : s.hi[d];
      }
      any = true;
    }
    if (any) push_box(v, x, x, h);
  }
  return v;
}

int build_xfers(amss_engine* e) {
  e->xfers.clear();
  e->staging.clear();
  for (auto& kv : e->levels) {
    ELevel& L = kv.second;
    L.xsync = plan_xfer(e, XF_SYNC, kv.first, sync_boxes(e, L));
    if (kv.first > 0) {
      ELevel& C = e->levels[kv.first - 1];
      L.xrestrict = plan_xfer(e, XF_RESTRICT, kv.first, restrict_boxes(e, L, C));
      L.xprolong = plan_xfer(e, XF_PROLONG, kv.first, prolong_boxes(e, L, C));
    }
  }
  e->stage_out_bytes = e->stage_in_bytes = 0;
  for (const XferOp& op : e->xfers) {
    e->stage_out_bytes = std::max(e->stage_out_bytes, op.out_bytes);
    e->stage_in_bytes = std::max(e->stage_in_bytes, op.in_bytes);
  }
  return 0;
}

int upload_xfers(amss_engine* e, std::vector<AmrBlock>& table) {
  if (e->stage_out_bytes) AMSS_CK(cudaMalloc(&e->stage_out, e->stage_out_bytes));
  if (e->stage_in_bytes) AMSS_CK(cudaMalloc(&e->stage_in, e->stage_in_bytes));
  const bool mixed = e->prm.precision == 1;
  for (const XStage& s : e->staging) {
    AmrBlock a{};
    for (int d = 0; d < 3; ++d) { a.org[d] = s.org[d]; a.ex[d] = s.ex[d]; }
    const long long n = (long long)s.ex[0] * s.ex[1] * s.ex[2];
    a.fs = n;
    char* base = (s.in ? e->stage_in : e->stage_out) + s.off;
    for (int t = 0; t < 3; ++t) a.tl[t] = (double*)base;
    a.K = (double*)base;
    a.st[0] = a.st[1] = base;
    if (mixed) a.side[0] = a.side[1] = (double*)(base + align256((long long)e->nf * n * 4));
    a.lvl = e->dlvl;   // every time level is the same region: the ring index does not matter
    a.nf = e->nf;
    table.push_back(a);
  }
  for (XferOp& op : e->xfers) {
    if (int rc = upload_boxes(op.run_h, op.run, op.kind == XF_SYNC ? 0 : e->nf, op.kind == XF_PROLONG)) return rc;
    if (int rc = upload_boxes(op.unpack_h, op.unpack)) return rc;
  }
  return 0;
}

void release_xfers(amss_engine* e) {
  for (XferOp& op : e->xfers) {
    op.run.release();
    op.unpack.release();
  }
  if (e->stage_out) cudaFree(e->stage_out);
  if (e->stage_in) cudaFree(e->stage_in);
  e->stage_out = e->stage_in = nullptr;
  if (e->ev_ready) cudaEventDestroy(e->ev_ready);
  if (e->ev_done) cudaEventDestroy(e->ev_done);
  e->ev_ready = e->ev_done = nullptr;
}

// ---- transports ---------------------------------------------------------------

static int group_barrier(amss_group* g) {
  std::unique_lock<std::mutex> lk(g->mu);
  if (g->broken) return amss_fail(AMSS_ERR_STATE, "rank group: a rank failed or timed out at an earlier exchange");
  const long long my = g->gen;
  if (++g->arrived == g->n) {
    g->arrived = 0;
    g->gen++;
    g->cv.notify_all();
    return 0;
  }
  const auto limit = std::chrono::duration<double>(g->timeout_s);
  const bool ok = g->cv.wait_for(lk, limit, [&] { return g->gen != my || g->broken; });
  if (!ok || g->gen == my) {
    g->broken = true;
    g->cv.notify_all();
    return amss_fail(AMSS_ERR_STATE, "rank group: not every rank reached the exchange within the timeout");
  }
  return 0;
}

static const XPeer* find_peer(const std::vector<XPeer>& v, int rank) {
  for (const XPeer& p : v)
    if (p.rank == rank) return &p;
  return nullptr;
}

static int group_exchange(amss_engine* e, int k) {
  amss_group* g = e->group;
  AMSS_CK(cudaEventRecord(e->ev_ready, e->stream));
  if (int rc = group_barrier(g)) return rc;
  const XferOp& op = e->xfers[k];
  int bad = 0;
  for (const XPeer& r : op.recv) {
    const amss_engine* p = g->eng[r.rank];
    const XPeer* s = k < (int)p->xfers.size() ? find_peer(p->xfers[k].send, e->rank) : nullptr;
    if (!s || s->bytes != r.bytes) { bad = 1; break; }
    if (cudaStreamWaitEvent(e->stream, p->ev_ready, 0) != cudaSuccess ||
        cudaMemcpyAsync(e->stage_in + r.off, p->stage_out + s->off, (size_t)r.bytes, cudaMemcpyDeviceToDevice,
                        e->stream) != cudaSuccess) { bad = 2; break; }
  }
  if (!bad && cudaEventRecord(e->ev_done, e->stream) != cudaSuccess) bad = 2;
  if (int rc = group_barrier(g)) return rc;   // met even after a failure, so the others do not wait out the timeout
  if (bad == 1) return amss_fail(AMSS_ERR_STATE, "rank group: the ranks' transfer plans disagree (same hierarchy and owners?)");
  if (bad == 2) return amss_fail(AMSS_ERR_CUDA, "rank group: device-to-device copy from a peer failed");
  for (const XPeer& s : op.send) AMSS_CK(cudaStreamWaitEvent(e->stream, g->eng[s.rank]->ev_done, 0));
  return 0;
}

struct NcclApi {
  ncclResult_t (*GetUniqueId)(ncclUniqueId*);
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int);
  ncclResult_t (*CommDestroy)(ncclComm_t);
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*GroupStart)();
  ncclResult_t (*GroupEnd)();
  const char* (*GetErrorString)(ncclResult_t);
};

// The NCCL already loaded in the process (PyTorch's) when there is one, else
// the first libnccl the loader finds.
static const NcclApi* nccl_api() {
  static NcclApi api;
  static int state = 0;   // 0 not tried, 1 ok, -1 missing
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (state) return state > 0 ? &api : nullptr;
  state = -1;
  void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h) return nullptr;
#define AMSS_SYM(field, name) api.field = (decltype(api.field))dlsym(h, name); if (!api.field) return nullptr
  AMSS_SYM(GetUniqueId, "ncclGetUniqueId");
  AMSS_SYM(CommInitRank, "ncclCommInitRank");
  AMSS_SYM(CommDestroy, "ncclCommDestroy");
  AMSS_SYM(Send, "ncclSend");
  AMSS_SYM(Recv, "ncclRecv");
  AMSS_SYM(GroupStart, "ncclGroupStart");
  AMSS_SYM(GroupEnd, "ncclGroupEnd");
  AMSS_SYM(GetErrorString, "ncclGetErrorString");
#undef AMSS_SYM
  state = 1;
  return &api;
}

static int nccl_fail(const NcclApi* A, ncclResult_t r, const char* what) {
  std::string m = std::string(what) + ": " + A->GetErrorString(r);
  return amss_fail(AMSS_ERR_CUDA, m.c_str());
}

static int nccl_exchange(amss_engine* e, int k) {
  const NcclApi* A = nccl_api();
  const XferOp& op = e->xfers[k];
  if (op.send.empty() && op.recv.empty()) return 0;
  ncclComm_t comm = (ncclComm_t)e->nccl;
  ncclResult_t r = A->GroupStart();
  if (r != ncclSuccess) return nccl_fail(A, r, "ncclGroupStart");
  for (const XPeer& s : op.send)
    if ((r = A->Send(e->stage_out + s.off, (size_t)s.bytes, ncclUint8, s.rank, comm, e->stream)) != ncclSuccess) break;
  if (r == ncclSuccess)
    for (const XPeer& q : op.recv)
      if ((r = A->Recv(e->stage_in + q.off, (size_t)q.bytes, ncclUint8, q.rank, comm, e->stream)) != ncclSuccess) break;
  const ncclResult_t r2 = A->GroupEnd();
  if (r != ncclSuccess) return nccl_fail(A, r, "ncclSend/ncclRecv");
  if (r2 != ncclSuccess) return nccl_fail(A, r2, "ncclGroupEnd");
  return 0;
}

int run_xfer(amss_engine* e, int k, int arg) {
  if (k < 0) return 0;
  XferOp& op = e->xfers[k];
  const bool mixed = e->prm.precision == 1;
  if (op.run.ntiles) {
    cudaError_t err = cudaSuccess;
    if (op.kind == XF_SYNC)
      err = launch_amr_sync(e->dblocks, op.run.boxes, op.run.tiles, op.run.ntiles, arg, mixed, e->dstatus, e->stream);
    else if (op.kind == XF_RESTRICT)
      err = launch_amr_restrict(e->dblocks, op.run.boxes, op.run.tiles, op.run.ntiles, arg, e->dstatus, e->stream);
    else
      err = launch_amr_prolong(e->dblocks, op.run.boxes, op.run.tiles, op.run.ntiles, arg, e->dstatus, e->stream);
    AMSS_CK(err);
    e->launches++;
  }
  if (op.ncross == 0) return 0;   // the same on every rank: all ranks skip the exchange together
  if (e->group) {
    if (int rc = group_exchange(e, k)) return rc;
  } else if (e->nccl) {
    if (int rc = nccl_exchange(e, k)) return rc;
  } else {
    return amss_fail(AMSS_ERR_STATE, "engine holds one rank's blocks but has no transport (amss_group_join or amss_engine_set_nccl)");
  }
  if (op.unpack.ntiles) {
    // the restriction wrote the parent's state or its time-interpolated
    // accumulator; the prolongation the child's state
    const int which = op.kind == XF_SYNC ? arg : op.kind == XF_RESTRICT ? (arg ? BUF_TEMP : BUF_STATE) : BUF_STATE;
    AMSS_CK(launch_amr_sync(e->dblocks, op.unpack.boxes, op.unpack.tiles, op.unpack.ntiles, which, mixed, e->dstatus,
                            e->stream));
    e->launches++;
  }
  return 0;
}

}  // namespace amss

using namespace amss;

// ---- C ABI ------------------------------------------------------------------

extern "C" amss_group* amss_group_create(int nranks, double timeout_s) {
  if (nranks < 1 || !(timeout_s > 0)) {
    amss_fail(AMSS_ERR_ARG, "amss_group_create: nranks >= 1 and a positive timeout");
    return nullptr;
  }
  amss_group* g = new amss_group();
  g->n = nranks;
  g->eng.assign(nranks, nullptr);
  g->timeout_s = timeout_s;
  return g;
}

extern "C" void amss_group_destroy(amss_group* g) { delete g; }

extern "C" int amss_group_barrier(amss_group* g) {
  if (!g) return amss_fail(AMSS_ERR_ARG, "amss_group_barrier: null group");
  return group_barrier(g);
}

extern "C" int amss_group_join(amss_engine* e, amss_group* g) {
  if (!e || !g || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "amss_group_join: commit the engine first");
  if (e->nranks != g->n) return amss_fail(AMSS_ERR_ARG, "amss_group_join: the group's size differs from the engine's nranks");
  if (e->nccl) return amss_fail(AMSS_ERR_STATE, "amss_group_join: the engine already uses NCCL");
  std::lock_guard<std::mutex> lk(g->mu);
  if (g->eng[e->rank]) return amss_fail(AMSS_ERR_STATE, "amss_group_join: the rank has joined already");
  g->eng[e->rank] = e;
  e->group = g;
  return 0;
}

extern "C" int amss_nccl_unique_id(unsigned char* out) {
  if (!out) return amss_fail(AMSS_ERR_ARG, "amss_nccl_unique_id: null buffer");
  const NcclApi* A = nccl_api();
  if (!A) return amss_fail(AMSS_ERR_UNSUPPORTED, "amss_nccl_unique_id: libnccl.so.2 could not be loaded");
  ncclUniqueId id;
  const ncclResult_t r = A->GetUniqueId(&id);
  if (r != ncclSuccess) return nccl_fail(A, r, "ncclGetUniqueId");
  std::memcpy(out, id.internal, NCCL_UNIQUE_ID_BYTES);
  return 0;
}

extern "C" int amss_engine_set_nccl(amss_engine* e, const unsigned char* uid) {
  if (!e || !uid || !e->committed || e->plan_only) return amss_fail(AMSS_ERR_STATE, "amss_engine_set_nccl: commit the engine first");
  if (e->group || e->nccl) return amss_fail(AMSS_ERR_STATE, "amss_engine_set_nccl: the engine has a transport already");
  const NcclApi* A = nccl_api();
  if (!A) return amss_fail(AMSS_ERR_UNSUPPORTED, "amss_engine_set_nccl: libnccl.so.2 could not be loaded");
  ncclUniqueId id;
  std::memcpy(id.internal, uid, NCCL_UNIQUE_ID_BYTES);
  ncclComm_t comm = nullptr;
  const ncclResult_t r = A->CommInitRank(&comm, e->nranks, id, e->rank);
  if (r != ncclSuccess) return nccl_fail(A, r, "ncclCommInitRank");
  e->nccl = comm;
  return 0;
}

void amss::amss_xfer_detach(amss_engine* e) {
  if (e->nccl) {
    const NcclApi* A = nccl_api();
    if (A) A->CommDestroy((ncclComm_t)e->nccl);
    e->nccl = nullptr;
  }
  if (e->group) {
    std::lock_guard<std::mutex> lk(e->group->mu);
    if (e->group->eng[e->rank] == e) e->group->eng[e->rank] = nullptr;
    e->group = nullptr;
  }
}

extern "C" int amss_engine_xfer_count(amss_engine* e) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  return (int)e->xfers.size();
}

extern "C" int amss_engine_xfer_info(amss_engine* e, int k, long long* info) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  if (k < 0 || k >= (int)e->xfers.size() || !info) return amss_fail(AMSS_ERR_ARG, "amss_engine_xfer_info: bad transfer");
  const XferOp& op = e->xfers[k];
  const long long v[8] = {op.kind, op.level, op.nall, op.ncross, (long long)op.run_h.size(),
                          (long long)op.unpack_h.size(), op.out_bytes, op.in_bytes};
  std::memcpy(info, v, sizeof v);
  return 0;
}

extern "C" int amss_engine_xfer_boxes(amss_engine* e, int k, int list, int* out, int cap) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  if (k < 0 || k >= (int)e->xfers.size() || (list != 0 && list != 1)) return amss_fail(AMSS_ERR_ARG, "amss_engine_xfer_boxes: bad transfer or list");
  const std::vector<AmrBox>& v = list == 0 ? e->xfers[k].run_h : e->xfers[k].unpack_h;
  if (!out) return (int)v.size();
  if (cap < (int)v.size()) return amss_fail(AMSS_ERR_ARG, "amss_engine_xfer_boxes: buffer too small");
  for (size_t i = 0; i < v.size(); ++i) {
    const AmrBox& b = v[i];
    const int r[8] = {b.dst, b.src, b.lo[0], b.lo[1], b.lo[2], b.n[0], b.n[1], b.n[2]};
    std::memcpy(out + 8 * i, r, sizeof r);
  }
  return (int)v.size();
}

extern "C" int amss_engine_xfer_peers(amss_engine* e, int k, int dir, long long* out, int cap) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  if (k < 0 || k >= (int)e->xfers.size() || (dir != 0 && dir != 1)) return amss_fail(AMSS_ERR_ARG, "amss_engine_xfer_peers: bad transfer or direction");
  const std::vector<XPeer>& v = dir == 0 ? e->xfers[k].send : e->xfers[k].recv;
  if (!out) return (int)v.size();
  if (cap < (int)v.size()) return amss_fail(AMSS_ERR_ARG, "amss_engine_xfer_peers: buffer too small");
  for (size_t i = 0; i < v.size(); ++i) {
    out[3 * i] = v[i].rank;
    out[3 * i + 1] = v[i].off;
    out[3 * i + 2] = v[i].bytes;
  }
  return (int)v.size();
}

extern "C" int amss_engine_staging_block(amss_engine* e, int id, long long* out) {
  if (!e || !e->committed) return amss_fail(AMSS_ERR_STATE, "engine not committed");
  const int i = id - (int)e->blocks.size();
  if (i < 0 || i >= (int)e->staging.size() || !out) return amss_fail(AMSS_ERR_ARG, "amss_engine_staging_block: not a staging block");
  const XStage& s = e->staging[i];
  const long long v[8] = {s.org[0], s.org[1], s.org[2], s.ex[0], s.ex[1], s.ex[2], s.off, s.in};
  std::memcpy(out, v, sizeof v);
  return 0;
}
