// Instantiations and launch entry points of the importance-sampling kernels.
#include "sim_is.cuh"

namespace csmc {

size_t is_mlp_smem_bytes() { return sizeof(detail::MlpSmem); }

template <bool TC, bool TRACE, bool SLOTS>
static int is_launch_l(bool loc8, const IsParams &p, int grid, int block, size_t smem, void *stream) {
    return loc8 ? is_launch_one<TC, TRACE, SLOTS, true>(p, grid, block, smem, stream)
                : is_launch_one<TC, TRACE, SLOTS, false>(p, grid, block, smem, stream);
}

template <bool TC>
static int is_launch_t(bool trace, bool slots, bool loc8, const IsParams &p, int grid, int block, size_t smem,
                       void *stream) {
    if (trace) return slots ? is_launch_l<TC, true, true>(loc8, p, grid, block, smem, stream)
                            : is_launch_l<TC, true, false>(loc8, p, grid, block, smem, stream);
    return slots ? is_launch_l<TC, false, true>(loc8, p, grid, block, smem, stream)
                 : is_launch_l<TC, false, false>(loc8, p, grid, block, smem, stream);
}

int is_launch(bool tc, bool trace, bool slots, bool loc8, const IsParams &p, int grid, int block, size_t smem,
              void *stream) {
    return tc ? is_launch_t<true>(trace, slots, loc8, p, grid, block, smem, stream)
              : is_launch_t<false>(trace, slots, loc8, p, grid, block, smem, stream);
}

template <bool TC, bool TRACE, bool SLOTS>
static int is_occ_l(bool loc8, int block, size_t smem, int *ctas) {
    return loc8 ? is_occupancy_one<TC, TRACE, SLOTS, true>(block, smem, ctas)
                : is_occupancy_one<TC, TRACE, SLOTS, false>(block, smem, ctas);
}

template <bool TC>
static int is_occ_t(bool trace, bool slots, bool loc8, int block, size_t smem, int *ctas) {
    if (trace) return slots ? is_occ_l<TC, true, true>(loc8, block, smem, ctas) : is_occ_l<TC, true, false>(loc8, block, smem, ctas);
    return slots ? is_occ_l<TC, false, true>(loc8, block, smem, ctas) : is_occ_l<TC, false, false>(loc8, block, smem, ctas);
}

int is_max_active_ctas(bool tc, bool trace, bool slots, bool loc8, int block, size_t smem, int *ctas) {
    return tc ? is_occ_t<true>(trace, slots, loc8, block, smem, ctas)
              : is_occ_t<false>(trace, slots, loc8, block, smem, ctas);
}

}  // namespace csmc
