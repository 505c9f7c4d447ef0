// Dispatch from a runtime (lanes per run, components per lane) shape to the
// kernel instantiations in sim_shapes_*.cu.
#include "sim.cuh"

#include <cuda_runtime.h>

namespace csmc {

template <int G, int K, bool VERIFY>
int launch_one(const SimParams &p, int grid, int block, size_t smem, void *stream);
template <int G, int K, bool VERIFY>
int occupancy_one(int block, size_t smem, int *ctas);
template <bool VERIFY, bool SLOTS, bool LOC8, bool GSTATE, bool CLASSES>
int serial_launch_one(const SimParams &p, int grid, int block, size_t smem, void *stream);
template <bool VERIFY, bool SLOTS, bool LOC8, bool GSTATE, bool CLASSES>
int serial_occupancy_one(int block, size_t smem, int *ctas);

// 32 instantiations, selected by five run-time flags
template <bool V, bool S, bool L, bool G>
static int serial_launch_c(bool classes, const SimParams &p, int grid, int block, size_t smem, void *stream) {
    return classes ? serial_launch_one<V, S, L, G, true>(p, grid, block, smem, stream)
                   : serial_launch_one<V, S, L, G, false>(p, grid, block, smem, stream);
}
template <bool V, bool S, bool L>
static int serial_launch_g(bool gstate, bool classes, const SimParams &p, int grid, int block, size_t smem,
                           void *stream) {
    return gstate ? serial_launch_c<V, S, L, true>(classes, p, grid, block, smem, stream)
                  : serial_launch_c<V, S, L, false>(classes, p, grid, block, smem, stream);
}
template <bool V, bool S>
static int serial_launch_l(bool loc8, bool gstate, bool classes, const SimParams &p, int grid, int block, size_t smem,
                           void *stream) {
    return loc8 ? serial_launch_g<V, S, true>(gstate, classes, p, grid, block, smem, stream)
                : serial_launch_g<V, S, false>(gstate, classes, p, grid, block, smem, stream);
}
int serial_launch(bool verify, bool slots, bool loc8, bool gstate, bool classes, const SimParams &p, int grid,
                  int block, size_t smem, void *stream) {
    if (verify) return slots ? serial_launch_l<true, true>(loc8, gstate, classes, p, grid, block, smem, stream)
                             : serial_launch_l<true, false>(loc8, gstate, classes, p, grid, block, smem, stream);
    return slots ? serial_launch_l<false, true>(loc8, gstate, classes, p, grid, block, smem, stream)
                 : serial_launch_l<false, false>(loc8, gstate, classes, p, grid, block, smem, stream);
}

template <bool V, bool S, bool L, bool G>
static int serial_occ_c(bool classes, int block, size_t smem, int *ctas) {
    return classes ? serial_occupancy_one<V, S, L, G, true>(block, smem, ctas)
                   : serial_occupancy_one<V, S, L, G, false>(block, smem, ctas);
}
template <bool V, bool S, bool L>
static int serial_occ_g(bool gstate, bool classes, int block, size_t smem, int *ctas) {
    return gstate ? serial_occ_c<V, S, L, true>(classes, block, smem, ctas)
                  : serial_occ_c<V, S, L, false>(classes, block, smem, ctas);
}
template <bool V, bool S>
static int serial_occ_l(bool loc8, bool gstate, bool classes, int block, size_t smem, int *ctas) {
    return loc8 ? serial_occ_g<V, S, true>(gstate, classes, block, smem, ctas)
                : serial_occ_g<V, S, false>(gstate, classes, block, smem, ctas);
}
int serial_max_active_ctas(bool verify, bool slots, bool loc8, bool gstate, bool classes, int block, size_t smem,
                           int *ctas) {
    if (verify) return slots ? serial_occ_l<true, true>(loc8, gstate, classes, block, smem, ctas)
                             : serial_occ_l<true, false>(loc8, gstate, classes, block, smem, ctas);
    return slots ? serial_occ_l<false, true>(loc8, gstate, classes, block, smem, ctas)
                 : serial_occ_l<false, false>(loc8, gstate, classes, block, smem, ctas);
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
