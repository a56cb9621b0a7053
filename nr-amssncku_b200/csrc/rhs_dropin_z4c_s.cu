// Instantiation of the drop-in Z4c RHS kernel, symmetry planes yes.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_rhs_dropin_z4c<true>(int, cudaStream_t, BlockView, Coefs<double>, const double*, double*,
                                                const double*, unsigned*);
}  // namespace amss
