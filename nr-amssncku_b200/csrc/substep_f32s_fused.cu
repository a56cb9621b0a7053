// Instantiation of the RK4 substep kernels: arithmetic float, stage storage float, symmetry planes yes,
// fused (one pass) form.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_substep<float, float, true, false, false>(const void*, const int2*, int, int, RKConst, int,
                                                       unsigned*, int, cudaStream_t, const void*, long long);
template cudaError_t launch_face<float, float, true>(const void*, const int2*, int, int, RKConst, int, unsigned*,
                                                cudaStream_t);
}  // namespace amss
