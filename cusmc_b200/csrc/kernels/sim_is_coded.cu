// Instantiations and launch entry points of the thread-per-run
// importance-sampling kernel.
#include "sim_is_coded.cuh"

namespace csmc {

int is_coded_launch(bool slots, bool all_grouped, const IsParams &p, int grid, int block, size_t smem, void *stream) {
    if (all_grouped)
        return slots ? is_coded_launch_one<true, true>(p, grid, block, smem, stream)
                     : is_coded_launch_one<false, true>(p, grid, block, smem, stream);
    return slots ? is_coded_launch_one<true, false>(p, grid, block, smem, stream)
                 : is_coded_launch_one<false, false>(p, grid, block, smem, stream);
}

size_t is_coded_mlp_smem_bytes() { return detail::kMlpExactBytes; }
size_t is_coded_warp_smem_bytes() { return 4u * detail::kThetaBatch * CSMC_MLP_HID * CSMC_MLP_CLASSES; }

int is_coded_max_active_ctas(bool slots, bool all_grouped, int block, size_t smem, int *ctas) {
    if (all_grouped)
        return slots ? is_coded_occupancy_one<true, true>(block, smem, ctas)
                     : is_coded_occupancy_one<false, true>(block, smem, ctas);
    return slots ? is_coded_occupancy_one<true, false>(block, smem, ctas)
                 : is_coded_occupancy_one<false, false>(block, smem, ctas);
}

}  // namespace csmc
