// Instantiation of the fused RK4 substep: arithmetic float, stage storage float, symmetry planes yes.
#include "substep_impl.cuh"

namespace amss {
template cudaError_t launch_substep<float, float, true>(const void*, const int2*, int, int, RKConst, int, unsigned*, int,
                                                   cudaStream_t);
}  // namespace amss
