// Thread-per-run simulation kernel for one network.
//
// Every thread simulates one run at a time and walks that run's components
// in a loop, so a warp advances 32 independent runs in lockstep through the
// same instruction stream: no shuffles, no warp barriers, and the winner's
// transition is executed by all 32 lanes for their own runs at once.  A lane
// whose run ends takes the next run index from the device work counter
// immediately (warp-aggregated atomic), so uneven run lengths do not idle the
// warp.  The run state and the step are those of sim_run.cuh.
//
// Template options: SLOTS keeps the slot masks; LOC8 stores locations as
// 8-bit local indices (automata of at most 256 locations), otherwise as
// 16-bit global indices; GSTATE puts the state in per-CTA global slabs when
// it does not fit in shared memory; CLASSES decides the race from race
// classes (sim_run.cuh: race_classes).  The network layout comes from the
// kernel parameters, so pointers into the staged network are rebuilt from
// constants instead of occupying registers.
//
// Reference: simulation/simulation.cu:674-901 (simulation_kernel).
#pragma once
#include "sim_run.cuh"

namespace csmc {
namespace detail {

#ifndef CSMC_SERIAL_MIN_CTAS_PER_SM
#define CSMC_SERIAL_MIN_CTAS_PER_SM 4
#endif

template <bool VERIFY, bool SLOTS, bool LOC8, bool GSTATE, bool CLASSES>
__global__ void __launch_bounds__(128, CSMC_SERIAL_MIN_CTAS_PER_SM) serial_kernel(const SimParams p) {
    extern __shared__ __align__(16) uint8_t smem[];
    stage_network(smem, p.blob, p.blob_bytes);
    __syncthreads();
    const Net n = net_view(smem, p.net);
    const uint32_t C = p.net.n_comps, V = p.net.n_vars, P = p.net.n_rate_prog;
    const bool rate_table = (p.net.flags & CSMC_NET_RATE_TABLE) && P > 0;

    // per-thread interleaved state
    const uint32_t T = blockDim.x, t = threadIdx.x;
    uint8_t *st = GSTATE ? p.state_global + static_cast<size_t>(blockIdx.x) * p.state_stride : smem + p.blob_bytes;
    const RunView<LOC8> rv = carve_run_view<LOC8>(st, V, P, C, T, t);

    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;

    bool have = false;
    unsigned long long ridx = 0;
    uint64_t run = 0;
    float time = 0.0f;
    uint32_t step = 0;
    RunScalars sc{0.0, 0.0, 0, 0, -1, 0, 0};

    for (;;) {
        // ---- refill finished lanes from the work counter
        const bool need = !have;
        const unsigned act = __activemask();
        const unsigned want = __ballot_sync(act, need);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if (static_cast<int>(lane) == leader)
                base = atomicAdd(p.scratch, static_cast<unsigned long long>(__popc(want)));
            base = __shfl_sync(act, base, leader);
            if (need) {
                ridx = base + __popc(want & ((1u << lane) - 1u));
                if (ridx >= p.n_runs) break;
                have = true;
                run = p.first_run + ridx;
                run_init<SLOTS>(n, C, V, rv, sc, p.var_id);
                time = 0.0f;
                step = 0;
            }
        }

        // ---- end of run (simulation.cu:835-849, 887-893)
        const RunEnd e = run_end(sc, time, p.horizon, step, p.max_steps, p.loc_mode, p.is_max, p.threshold);
        if (e.done) {
            if (p.flags) p.flags[ridx] = static_cast<uint8_t>(e.flag);
            if (p.values) p.values[ridx] = e.value;
            if (p.steps) p.steps[ridx] = step;
            if (VERIFY) {
                if (p.digests) p.digests[ridx] = sc.digest;
                if (p.final_state) run_final_state(n, C, V, rv, p.final_state + ridx * (C + V));
            }
            acc_hits += e.flag;
            acc_steps += step;
            acc_capped += e.capped;
            have = false;
            continue;
        }

        run_step<VERIFY, SLOTS, CLASSES>(n, C, V, P, p.net.n_clocks, rate_table, rv, sc, p.seed, p.var_id, run,
                                               step, time);
    }
    // lanes leave the loop at different times; aggregate per lane
    if (acc_hits) atomicAdd(p.scratch + 1, acc_hits);
    if (acc_steps) atomicAdd(p.scratch + 2, acc_steps);
    if (acc_capped) atomicAdd(p.scratch + 3, acc_capped);
}

}  // namespace detail

template <bool VERIFY, bool SLOTS, bool LOC8, bool GSTATE, bool CLASSES>
int serial_launch_one(const SimParams &p, int grid, int block, size_t smem, void *stream) {
    auto fn = detail::serial_kernel<VERIFY, SLOTS, LOC8, GSTATE, CLASSES>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool VERIFY, bool SLOTS, bool LOC8, bool GSTATE, bool CLASSES>
int serial_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::serial_kernel<VERIFY, SLOTS, LOC8, GSTATE, CLASSES>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
