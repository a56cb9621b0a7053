// Instantiation of the RK4 substep kernels for Z4c: arithmetic float, stage storage float,
// symmetry planes yes, split (stencil pass + pointwise pass) form.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_substep<float, float, true, true, true>(const void*, const int2*, int, int, RKConst, int,
                                                       unsigned*, int, cudaStream_t, const void*, long long);
}  // namespace amss
