// Kernel instantiations for lane-group shapes: 32,16
#include "sim_impl.cuh"

namespace csmc {
CSMC_INSTANTIATE_SHAPE(32, 16)
}  // namespace csmc
