// Instantiations and launch entry points of the thread-per-run
// importance-sampling kernel.
#include "sim_is_coded.cuh"

namespace csmc {

int is_coded_launch(bool slots, const IsParams &p, int grid, int block, size_t smem, void *stream) {
    return slots ? is_coded_launch_one<true>(p, grid, block, smem, stream)
                 : is_coded_launch_one<false>(p, grid, block, smem, stream);
}

size_t is_coded_mlp_smem_bytes() { return detail::kMlpExactBytes; }
size_t is_coded_warp_smem_bytes() { return 4u * detail::kThetaBatch * CSMC_MLP_HID * CSMC_MLP_CLASSES; }

int is_coded_max_active_ctas(bool slots, int block, size_t smem, int *ctas) {
    return slots ? is_coded_occupancy_one<true>(block, smem, ctas) : is_coded_occupancy_one<false>(block, smem, ctas);
}

}  // namespace csmc
