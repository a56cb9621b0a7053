// Instantiation of the RK4 substep kernels: arithmetic float, stage storage float, symmetry planes no,
// fused (one pass) form.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_substep<float, float, false, false, false>(const void*, const int2*, int, int, RKConst, int,
                                                       unsigned*, int, cudaStream_t, const void*, long long);
template cudaError_t launch_face<float, float, false>(const void*, const int2*, int, int, RKConst, int, unsigned*,
                                                cudaStream_t);
}  // namespace amss
