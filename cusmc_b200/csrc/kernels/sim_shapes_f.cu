// Kernel instantiations for lane-group shapes: 32,32
#include "sim_impl.cuh"

namespace csmc {
CSMC_INSTANTIATE_SHAPE(32, 32)
}  // namespace csmc
