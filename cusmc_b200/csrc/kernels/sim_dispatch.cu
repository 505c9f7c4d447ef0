// Dispatch from a runtime (lanes per run, components per lane) shape to the
// kernel instantiations in sim_shapes_*.cu.
#include "sim.cuh"

#include <cuda_runtime.h>

namespace csmc {

template <int G, int K, bool VERIFY>
int launch_one(const SimParams &p, int grid, int block, size_t smem, void *stream);
template <int G, int K, bool VERIFY>
int occupancy_one(int block, size_t smem, int *ctas);
template <bool VERIFY, bool SLOTS>
int serial_launch_one(const SimParams &p, int grid, int block, size_t smem, void *stream);
template <bool VERIFY, bool SLOTS>
int serial_occupancy_one(int block, size_t smem, int *ctas);

int serial_launch(bool verify, bool slots, const SimParams &p, int grid, int block, size_t smem, void *stream) {
    if (verify) return slots ? serial_launch_one<true, true>(p, grid, block, smem, stream)
                             : serial_launch_one<true, false>(p, grid, block, smem, stream);
    return slots ? serial_launch_one<false, true>(p, grid, block, smem, stream)
                 : serial_launch_one<false, false>(p, grid, block, smem, stream);
}

int serial_max_active_ctas(bool verify, bool slots, int block, size_t smem, int *ctas) {
    if (verify) return slots ? serial_occupancy_one<true, true>(block, smem, ctas)
                             : serial_occupancy_one<true, false>(block, smem, ctas);
    return slots ? serial_occupancy_one<false, true>(block, smem, ctas)
                 : serial_occupancy_one<false, false>(block, smem, ctas);
}

#define CSMC_SHAPES(X) X(1, 1) X(2, 1) X(4, 1) X(8, 1) X(16, 1) X(32, 1) X(32, 2) X(32, 4) X(32, 8) X(32, 16) X(32, 32)

bool sim_supported(int g, int k) {
#define X(GG, KK) \
    if (g == GG && k == KK) return true;
    CSMC_SHAPES(X)
#undef X
    return false;
}

int sim_launch(int g, int k, bool verify, const SimParams &p, int grid, int block, size_t smem, void *stream) {
#define X(GG, KK)                                                              \
    if (g == GG && k == KK)                                                    \
        return verify ? launch_one<GG, KK, true>(p, grid, block, smem, stream) \
                      : launch_one<GG, KK, false>(p, grid, block, smem, stream);
    CSMC_SHAPES(X)
#undef X
    return static_cast<int>(cudaErrorInvalidValue);
}

int sim_max_active_ctas(int g, int k, bool verify, int block, size_t smem, int *ctas) {
#define X(GG, KK)                                                    \
    if (g == GG && k == KK)                                          \
        return verify ? occupancy_one<GG, KK, true>(block, smem, ctas) \
                      : occupancy_one<GG, KK, false>(block, smem, ctas);
    CSMC_SHAPES(X)
#undef X
    return static_cast<int>(cudaErrorInvalidValue);
}

}  // namespace csmc
