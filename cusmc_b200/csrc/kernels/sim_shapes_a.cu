// Kernel instantiations for lane-group shapes: 1,1 2,1 4,1 8,1
#include "sim_impl.cuh"

namespace csmc {
CSMC_INSTANTIATE_SHAPE(1, 1)
CSMC_INSTANTIATE_SHAPE(2, 1)
CSMC_INSTANTIATE_SHAPE(4, 1)
CSMC_INSTANTIATE_SHAPE(8, 1)
}  // namespace csmc
