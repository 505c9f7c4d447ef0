// Instantiations and run-time dispatch of the class-coded thread-per-run
// kernel (sim_coded.cuh).
#include "sim_coded.cuh"

namespace csmc {

template <bool V, bool S>
static int coded_launch_a(bool all_classed, const SimParams &p, int grid, int block, size_t smem, void *stream) {
    return all_classed ? coded_launch_one<V, S, true>(p, grid, block, smem, stream)
                       : coded_launch_one<V, S, false>(p, grid, block, smem, stream);
}

int coded_launch(bool verify, bool slots, bool all_classed, const SimParams &p, int grid, int block, size_t smem,
                 void *stream) {
    if (verify) return slots ? coded_launch_a<true, true>(all_classed, p, grid, block, smem, stream)
                             : coded_launch_a<true, false>(all_classed, p, grid, block, smem, stream);
    return slots ? coded_launch_a<false, true>(all_classed, p, grid, block, smem, stream)
                 : coded_launch_a<false, false>(all_classed, p, grid, block, smem, stream);
}

template <bool V, bool S>
static int coded_occ_a(bool all_classed, int block, size_t smem, int *ctas) {
    return all_classed ? coded_occupancy_one<V, S, true>(block, smem, ctas)
                       : coded_occupancy_one<V, S, false>(block, smem, ctas);
}

int coded_max_active_ctas(bool verify, bool slots, bool all_classed, int block, size_t smem, int *ctas) {
    if (verify) return slots ? coded_occ_a<true, true>(all_classed, block, smem, ctas)
                             : coded_occ_a<true, false>(all_classed, block, smem, ctas);
    return slots ? coded_occ_a<false, true>(all_classed, block, smem, ctas)
                 : coded_occ_a<false, false>(all_classed, block, smem, ctas);
}

}  // namespace csmc
