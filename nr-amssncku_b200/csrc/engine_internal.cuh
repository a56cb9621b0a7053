// engine_internal.cuh -- host-side state of the batched engine, shared by
// engine.cu (blocks, tables, the level step) and xfer.cu (the transfer plans
// and their exchange between ranks).
#pragma once
#include <condition_variable>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "amr_types.cuh"
#include "deriv.cuh"
#include "dev_util.cuh"
#include "interp.cuh"

struct amss_group;

namespace amss {

struct Box {
  int lo[3], hi[3];
  bool empty() const { return lo[0] >= hi[0] || lo[1] >= hi[1] || lo[2] >= hi[2]; }
};
inline Box intersect(const Box& a, const Box& b) {
  Box r;
  for (int d = 0; d < 3; ++d) {
    r.lo[d] = a.lo[d] > b.lo[d] ? a.lo[d] : b.lo[d];
    r.hi[d] = a.hi[d] < b.hi[d] ? a.hi[d] : b.hi[d];
  }
  return r;
}

struct EPatch {
  int level;
  Box phys;            // physical cells
  int buffer;          // buffer cells each side (0 on level 0)
  Box ext() const {
    Box b = phys;
    for (int d = 0; d < 3; ++d) { b.lo[d] -= buffer; b.hi[d] += buffer; }
    return b;
  }
  std::vector<int> blocks;
};

struct EBlock {
  int level = 0, patch = -1;
  int owner = 0;                // rank that holds the block's arrays and steps it
  int ex[3], org[3];
  Box own;
  long long npts, fs;
  double bbox[6], pbbox[6];
  std::vector<double> X, Y, Z;
  int face_mask = 0, lowsym = 0;
  bool l2_by_bbox = false;      // added by bbox: its L2-norm cells follow l2normhelper's bbox test
  double* dX = nullptr;
  double* tl[3] = {nullptr, nullptr, nullptr};
  double* K = nullptr;
  void* st[2] = {nullptr, nullptr};
  double* side[2] = {nullptr, nullptr};
  Box array() const {
    Box b;
    for (int d = 0; d < 3; ++d) { b.lo[d] = org[d]; b.hi[d] = org[d] + ex[d]; }
    return b;
  }
};

struct DevBoxes {
  AmrBox* boxes = nullptr;
  int2* tiles = nullptr;
  int ntiles = 0;
  void release() {
    if (boxes) cudaFree(boxes);
    if (tiles) cudaFree(tiles);
    boxes = nullptr;
    tiles = nullptr;
  }
};

// One data movement between blocks of the hierarchy (the reference's
// Parallel::Sync, Restrict, OutBdLow2Hi) as one rank runs it.  The full box
// list is the same on every rank; a rank keeps the boxes whose source block it
// owns (`run`: computed by the transfer's kernel, into the destination block
// when it owns that too, else into a staging block that is sent to the
// destination's owner) and those whose destination it owns but not the
// source (`unpack`: a plain copy from the received staging block).  Staging
// blocks are extra entries of the AMR block table, after the real blocks:
// their array is the box, their buffers one region of the staging arena.
enum XferKind : int { XF_SYNC = 0, XF_RESTRICT = 1, XF_PROLONG = 2 };
struct XPeer {
  int rank;
  long long off, bytes;         // this rank's region of its staging arena for that peer
};
struct XStage {
  int org[3], ex[3];
  long long off;                // byte offset in the staging arena
  int in;                       // 0: staging-out arena, 1: staging-in
};
struct XferOp {
  int kind = XF_SYNC, level = 0;   // sync: the level; restrict / prolong: the fine level
  long long nall = 0;              // boxes of the transfer over all ranks
  long long ncross = 0;            // of which cross ranks (the same number on every rank)
  std::vector<AmrBox> run_h, unpack_h;
  DevBoxes run, unpack;
  std::vector<XPeer> send, recv;
  long long out_bytes = 0, in_bytes = 0;
};

struct ELevel {
  std::vector<int> blocks;      // every block of the level (all ranks)
  std::vector<int> own;         // the blocks this rank owns; the step tables index these
  std::vector<int> patches;
  int ntiles = 0;
  int2* dtiles = nullptr;       // substep tiles (index into this level's table)
  void* dtable = nullptr;       // StepBlock table
  bool symm = false;
  int xsync = -1, xrestrict = -1, xprolong = -1;   // transfers (index into amss_engine::xfers)
  int2* dti_tiles = nullptr;    // time-interpolation tiles (global block ids)
  int nti = 0;
  DevBoxes dti_boxes;           // the cells the next finer level's prolongation reads (timeinterp_boxes)
  int2* dfaces = nullptr;       // outer-face points (table index, point) for k_face
  int nfaces = 0;
  DerivItem* ditems = nullptr;  // stencil-pass work items (split form)
  int nditems = 0;
  // The final substep of a coarse step's level step over each block's owned
  // cells within final_pad of its patch's physical box (-1: whole arrays):
  // the cells further out are overwritten by the prolongation into the
  // level's buffer before anything reads them (plan_final_regions).
  int final_pad = -1;
  int2* dtiles_f = nullptr;     // region tiles of the final substep's pointwise pass
  int ntiles_f = 0;
  DerivItem* ditems_f = nullptr;   // and its stencil-pass items
  int nditems_f = 0;
  // The substeps over each block's owned cells only: the same-level sync
  // after every substep overwrites all of its ghost cells (plan_final_regions).
  bool own_ok = false;
  int2* dtiles_s = nullptr;     // owned-cell tiles of the pointwise pass
  int ntiles_s = 0;
  DerivItem* ditems_s = nullptr;   // and the stencil-pass items
  int nditems_s = 0;
  int tile_w = 0;               // stencil-pass tile width (0: deriv_tile_w of each block's x extent)
  int zsplit = 1;               // z-slabs per block in the stencil pass
  int docc = 0;                 // stencil-pass occupancy form: 0 two resident CTAs, 1 more (deriv.cuh)
  long long dfs = 0;            // slot stride of D for this level
  int* dregion = nullptr;       // per table block: local [lo, hi) of its owned cells inside its patch
  int* dregion_first = nullptr; // the same, empty for blocks outside the level's first patch
  int cur = 0;                  // host mirror of the ring index
  long long steps = 0;
};

}  // namespace amss

struct amss_engine {
  amss_params prm;
  bool grid_set = false;
  double x0[3] = {0, 0, 0};
  double h0 = 1.0;
  std::vector<amss::EBlock> blocks;
  std::vector<amss::EPatch> patches;
  std::map<std::pair<int, int>, int> patch_ids;   // (level, patch) -> index
  std::map<int, amss::ELevel> levels;
  cudaStream_t stream = nullptr;
  unsigned* dstatus = nullptr;
  int* dlvl = nullptr;          // 2 ints per level: ring index, steps taken
  amss::AmrBlock* dblocks = nullptr;   // AMR block table: the blocks, then the staging blocks
  void* D = nullptr;            // stencil terms of the level being stepped (split form)
  char* arena = nullptr;
  size_t arena_bytes = 0;
  long long launches = 0;
  bool committed = false;
  bool plan_only = false;       // built by amss_plan_create: transfer plans, no device state
  int sm_count = 148;
  int nf = amss::NFIELDS_BSSN;  // evolved fields: 24 (BSSN) or 25 (Z4c)
  double* cons = nullptr;       // constraint residuals of a level (7 x its D stride), grow-only
  long long cons_cap = 0;
  double* cpart = nullptr;      // per-CTA partial sums of the constraint norms (8 each)
  double* pscr = nullptr;       // Christoffel symbols and Ricci tensor of a level for Psi4 (24 x its D stride), grow-only
  long long pscr_cap = 0;
  int ntrack = 0, track_level = -1;   // puncture tracking on the finest level
  amss::TrackState* dtrack = nullptr;
  amss::TrackPatch* dtpatch = nullptr;
  amss::TrackBlock* dtblock = nullptr;
  int ntpatch = 0;
  amss::InterpItem* iitems = nullptr;   // point interpolation: items and results, grow-only
  double* iout = nullptr;
  long long icap = 0;
  // ranks: the blocks are divided among nranks engines, one per GPU
  int rank = 0, nranks = 1;
  std::vector<amss::XferOp> xfers;
  std::vector<amss::XStage> staging;   // staging blocks, table ids blocks.size() + i
  char* stage_out = nullptr;
  char* stage_in = nullptr;
  long long stage_out_bytes = 0, stage_in_bytes = 0;
  amss_group* group = nullptr;  // in-process ranks: peer engines, host barrier
  void* nccl = nullptr;         // ncclComm_t of the NCCL transport
  cudaEvent_t ev_ready = nullptr, ev_done = nullptr;
  int device = 0;               // the CUDA device the engine was created on
  bool owned(int b) const { return blocks[b].owner == rank; }
};

namespace amss {
// xfer.cu
int build_xfers(amss_engine* e);                       // host plans (every engine, plan-only included)
int upload_xfers(amss_engine* e, std::vector<AmrBlock>& table);   // staging arenas, blocks, device box lists
int run_xfer(amss_engine* e, int op, int arg);        // arg: sync buffer, restrict to_temp, prolong from_temp
void release_xfers(amss_engine* e);
void amss_xfer_detach(amss_engine* e);              // leaves its group, destroys its NCCL communicator
int upload_boxes(const std::vector<AmrBox>& boxes, DevBoxes& D, int nf = 0, bool runs = false);
// Sets each level's final_pad where the final-substep regions are safe, and
// own_ok where the same-level sync covers every ghost cell.
void plan_final_regions(amss_engine* e);
// Cells of C's blocks whose time interpolation F's prolongation reads.
std::vector<AmrBox> timeinterp_boxes(amss_engine* e, const ELevel& C, const ELevel& F);
// The final-substep region of a block (global level indices; empty: none).
Box final_region(const amss_engine* e, const ELevel& L, const EBlock& b);
void push_box(std::vector<AmrBox>& v, int dst, int src, const Box& b);
}  // namespace amss
