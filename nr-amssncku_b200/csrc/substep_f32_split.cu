// Instantiation of the RK4 substep kernels: arithmetic float, stage storage float, symmetry planes no,
// split (stencil pass + pointwise pass) form.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_substep<float, float, false, true, false>(const void*, const int2*, int, int, RKConst, int,
                                                       unsigned*, int, cudaStream_t, const void*, long long);
template cudaError_t launch_deriv<float, float>(const void*, const DerivItem*, int, int, void*, long long, int,
                                             cudaStream_t, int);
}  // namespace amss
