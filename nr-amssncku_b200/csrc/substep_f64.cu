// Instantiation of the fused RK4 substep: arithmetic double, stage storage double, symmetry planes no.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_substep<double, double, false>(const void*, const int2*, int, int, RKConst, int, unsigned*, int,
                                                   cudaStream_t);
}  // namespace amss
