// Instantiation of the drop-in RHS kernel, symmetry planes no.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_rhs_dropin<false>(int, cudaStream_t, BlockView, Coefs<double>, const double*, double*,
                                            RhsAux, unsigned*);
}  // namespace amss
