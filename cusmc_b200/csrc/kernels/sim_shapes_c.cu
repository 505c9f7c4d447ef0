// Kernel instantiations for lane-group shapes: 32,4
#include "sim_impl.cuh"

namespace csmc {
CSMC_INSTANTIATE_SHAPE(32, 4)
}  // namespace csmc
