// Instantiations and launch entry points of the multi-network batch kernel.
#include "sim_batch.cuh"

namespace csmc {

int batch_launch(bool verify, const BatchParams &p, int grid, int block, void *stream) {
    return verify ? batch_launch_one<true>(p, grid, block, stream) : batch_launch_one<false>(p, grid, block, stream);
}

int batch_max_active_ctas(bool verify, int block, size_t smem, int *ctas) {
    return verify ? batch_occupancy_one<true>(block, smem, ctas) : batch_occupancy_one<false>(block, smem, ctas);
}

}  // namespace csmc
