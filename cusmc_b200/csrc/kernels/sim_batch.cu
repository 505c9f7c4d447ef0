// Launch entry points of the multi-network batch kernel; the instantiations
// with warp-per-run jobs (K = 4, 8, 16 components per lane) are compiled in
// sim_batch_group.cu.
#include "sim_batch.cuh"

namespace csmc {

template <int K>
int batch_group_launch(bool verify, const BatchParams &p, int grid, int block, void *stream);
template <int K>
int batch_group_occupancy(bool verify, int block, size_t smem, int *ctas);

int batch_launch(bool verify, const BatchParams &p, int grid, int block, void *stream) {
    if (p.n_group_jobs == 0)
        return verify ? batch_launch_one<true, 0>(p, grid, block, stream)
                      : batch_launch_one<false, 0>(p, grid, block, stream);
    switch (p.group_k) {
        case 4: return batch_group_launch<4>(verify, p, grid, block, stream);
        case 8: return batch_group_launch<8>(verify, p, grid, block, stream);
        case 16: return batch_group_launch<16>(verify, p, grid, block, stream);
        default: return static_cast<int>(cudaErrorInvalidValue);
    }
}

int batch_max_active_ctas(bool verify, int group_k, int block, size_t smem, int *ctas) {
    switch (group_k) {
        case 0:
            return verify ? batch_occupancy_one<true, 0>(block, smem, ctas)
                          : batch_occupancy_one<false, 0>(block, smem, ctas);
        case 4: return batch_group_occupancy<4>(verify, block, smem, ctas);
        case 8: return batch_group_occupancy<8>(verify, block, smem, ctas);
        case 16: return batch_group_occupancy<16>(verify, block, smem, ctas);
        default: return static_cast<int>(cudaErrorInvalidValue);
    }
}

}  // namespace csmc
