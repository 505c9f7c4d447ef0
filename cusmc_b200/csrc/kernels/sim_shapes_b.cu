// Kernel instantiations for lane-group shapes: 16,1 32,1 32,2
#include "sim_impl.cuh"

namespace csmc {
CSMC_INSTANTIATE_SHAPE(16, 1)
CSMC_INSTANTIATE_SHAPE(32, 1)
CSMC_INSTANTIATE_SHAPE(32, 2)
}  // namespace csmc
