// Instantiation of the RK4 substep kernels: arithmetic double, stage storage double, symmetry planes no,
// split (stencil pass + pointwise pass) form.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_substep<double, double, false, true, false>(const void*, const int2*, int, int, RKConst, int,
                                                       unsigned*, int, cudaStream_t, const void*, long long);
template cudaError_t launch_deriv<double, double>(const void*, const DerivItem*, int, int, void*, long long, int,
                                             cudaStream_t, int);
}  // namespace amss
