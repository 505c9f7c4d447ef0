// Instantiations of the batch kernel with warp-per-run jobs (K components
// per lane).
#include "sim_batch.cuh"

namespace csmc {

template <int K>
int batch_group_launch(bool verify, const BatchParams &p, int grid, int block, void *stream) {
    return verify ? batch_launch_one<true, K>(p, grid, block, stream) : batch_launch_one<false, K>(p, grid, block, stream);
}

template <int K>
int batch_group_occupancy(bool verify, int block, size_t smem, int *ctas) {
    return verify ? batch_occupancy_one<true, K>(block, smem, ctas) : batch_occupancy_one<false, K>(block, smem, ctas);
}

template int batch_group_launch<4>(bool, const BatchParams &, int, int, void *);
template int batch_group_launch<8>(bool, const BatchParams &, int, int, void *);
template int batch_group_launch<16>(bool, const BatchParams &, int, int, void *);
template int batch_group_occupancy<4>(bool, int, size_t, int *);
template int batch_group_occupancy<8>(bool, int, size_t, int *);
template int batch_group_occupancy<16>(bool, int, size_t, int *);

}  // namespace csmc
