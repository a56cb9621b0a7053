// Instantiation of the RK4 substep kernels for Z4c: arithmetic double, stage storage double,
// symmetry planes yes, split (stencil pass + pointwise pass) form.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_substep<double, double, true, true, true>(const void*, const int2*, int, int, RKConst, int,
                                                       unsigned*, int, cudaStream_t, const void*, long long);
}  // namespace amss
