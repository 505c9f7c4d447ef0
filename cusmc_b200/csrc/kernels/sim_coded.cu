// Instantiations and run-time dispatch of the class-coded thread-per-run
// kernel (sim_coded.cuh).
#include "sim_coded.cuh"

namespace csmc {

int coded_launch(bool verify, bool slots, const SimParams &p, int grid, int block, size_t smem, void *stream) {
    if (verify) return slots ? coded_launch_one<true, true>(p, grid, block, smem, stream)
                             : coded_launch_one<true, false>(p, grid, block, smem, stream);
    return slots ? coded_launch_one<false, true>(p, grid, block, smem, stream)
                 : coded_launch_one<false, false>(p, grid, block, smem, stream);
}

int coded_max_active_ctas(bool verify, bool slots, int block, size_t smem, int *ctas) {
    if (verify) return slots ? coded_occupancy_one<true, true>(block, smem, ctas)
                             : coded_occupancy_one<true, false>(block, smem, ctas);
    return slots ? coded_occupancy_one<false, true>(block, smem, ctas)
                 : coded_occupancy_one<false, false>(block, smem, ctas);
}

}  // namespace csmc
