// Instantiation of the drop-in RHS kernel, symmetry planes yes.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_rhs_dropin<true>(int, cudaStream_t, BlockView, Coefs<double>, const double*, double*,
                                            RhsAux, unsigned*);
}  // namespace amss
