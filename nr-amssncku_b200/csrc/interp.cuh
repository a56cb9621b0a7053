// interp.cuh -- one (point, field) of the level interpolation: the field's
// current state array, the 6^3 stencil chosen by global_interp
// (fmisc.f90:738-781, Fortran indices, <= 0 means mirrored) and the point's
// offset from the stencil's first cell in cells.
#pragma once
#include <cuda_runtime.h>

namespace amss {

struct InterpItem {
  const double* f;   // one field of a block's current state (i fastest)
  int ex[3];
  int cxB[3];        // first stencil index per axis, Fortran numbering
  double cx[3];      // (x - X(cxB)) / dX per axis
  double soa[3];     // the field's parities
};

cudaError_t launch_interp_points(const InterpItem* items, int n, double* out, cudaStream_t s);

// Puncture tracking on the finest level.  A patch: its box less its buffer
// (the point search of Parallel::PatList_Interp_Points), half a cell, and
// its blocks [b0, b1) in the block table.
struct TrackPatch {
  double lo[3], hi[3], half[3];
  int b0, b1;
};
// A block: its state arrays (stages FP32 when f32), the box it answers for (Patch::Interp_Points),
// its cell-centre coordinates X(j) = blo + (j - 0.5) bh, X(1), X(2) - X(1),
// and the first stencil index allowed (-2 at a symmetry plane).
constexpr int kSideBetaX = 2;   // side slot of beta^x in the mixed form's FP64 stage fields (stencil.cuh)
struct TrackBlock {
  const double* tl[3];
  const void* stage[2];
  const double* side[2];   // FP64 side slots of the stages (mixed form: the shift is read there)
  long long fs;
  int ex[3], cmin[3], f32;
  double flo[3], fhi[3], blo[3], bh[3], x0[3], dd[3];
};
constexpr int kMaxPunctures = 10;
struct TrackState {
  double p0[3 * kMaxPunctures];     // Porg0: positions at the start of the step
  double pa[3 * kMaxPunctures];     // Porg: the estimates of substeps 0 and 2 ...
  double pb[3 * kMaxPunctures];     // ... and of substep 1
  double k[3 * kMaxPunctures];      // Porg_rhs: the RK4 accumulator
  int err;                          // a puncture left the finest level
};

cudaError_t launch_track(const TrackPatch* patches, int npatch, const TrackBlock* blocks, const int* lvl,
                         TrackState* S, int n, int sub, double dt, int symmetry, cudaStream_t s);

}  // namespace amss
