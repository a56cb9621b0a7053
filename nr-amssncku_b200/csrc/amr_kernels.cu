// amr_kernels.cu -- launch wrappers of the AMR data-movement kernels (amr.cuh).
#include "amr.cuh"
#include "dev_util.cuh"

namespace amss {

static int amr_grid(int ntiles) { return ntiles < 148 * 16 ? (ntiles < 1 ? 1 : ntiles) : 148 * 16; }

cudaError_t launch_amr_sync(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles, int which,
                            bool fp32_stages, unsigned* status, cudaStream_t s) {
  if (ntiles == 0) return cudaSuccess;
  if (fp32_stages && (which == BUF_STAGE_A || which == BUF_STAGE_B))
    k_amr_sync<float><<<amr_grid(ntiles), 128, 0, s>>>(blocks, boxes, tiles, ntiles, which, status);
  else
    k_amr_sync<double><<<amr_grid(ntiles), 128, 0, s>>>(blocks, boxes, tiles, ntiles, which, status);
  return cudaGetLastError();
}

cudaError_t launch_amr_prolong(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles,
                               int from_temp, unsigned* status, cudaStream_t s) {
  if (ntiles == 0) return cudaSuccess;
  k_amr_prolong<<<amr_grid(ntiles), 128, 0, s>>>(blocks, boxes, tiles, ntiles, from_temp, status);
  return cudaGetLastError();
}

cudaError_t launch_amr_restrict(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles,
                                int to_temp, unsigned* status, cudaStream_t s) {
  if (ntiles == 0) return cudaSuccess;
  k_amr_restrict<<<amr_grid(ntiles), 128, 0, s>>>(blocks, boxes, tiles, ntiles, to_temp, status);
  return cudaGetLastError();
}

cudaError_t launch_amr_timeinterp(const AmrBlock* blocks, const int2* tiles, int ntiles, cudaStream_t s) {
  if (ntiles == 0) return cudaSuccess;
  k_amr_timeinterp<<<amr_grid(ntiles), 128, 0, s>>>(blocks, tiles, ntiles);
  return cudaGetLastError();
}

cudaError_t launch_amr_timeinterp_boxes(const AmrBlock* blocks, const AmrBox* boxes, const int2* tiles, int ntiles,
                                        unsigned* status, cudaStream_t s) {
  if (ntiles == 0) return cudaSuccess;
  k_amr_timeinterp_boxes<<<amr_grid(ntiles), 128, 0, s>>>(blocks, boxes, tiles, ntiles, status);
  return cudaGetLastError();
}

cudaError_t launch_amr_enforce(const AmrBlock* blocks, const int2* tiles, int ntiles, cudaStream_t s) {
  if (ntiles == 0) return cudaSuccess;
  k_amr_enforce<<<amr_grid(ntiles), 128, 0, s>>>(blocks, tiles, ntiles);
  return cudaGetLastError();
}

cudaError_t launch_amr_rotate(int* lvl, cudaStream_t s) {
  k_amr_rotate<<<1, 1, 0, s>>>(lvl);
  return cudaGetLastError();
}

}  // namespace amss
