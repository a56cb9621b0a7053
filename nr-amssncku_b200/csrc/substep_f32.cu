// Instantiation of the fused RK4 substep: arithmetic float, stage storage float, symmetry planes no.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_substep<float, float, false>(const void*, const int2*, int, int, RKConst, int, unsigned*, int,
                                                   cudaStream_t);
}  // namespace amss
