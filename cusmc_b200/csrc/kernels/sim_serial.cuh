// Thread-per-run simulation kernel.
//
// Every thread simulates one run at a time and walks that run's components
// in a loop, so a warp advances 32 independent runs in lockstep through the
// same instruction stream: no shuffles, no warp barriers, and the winner's
// transition is executed by all 32 lanes for their own runs at once.  A lane
// whose run ends takes the next run index from the device work counter
// immediately (warp-aggregated atomic), so uneven run lengths do not idle the
// warp.  Per-run state lives in interleaved arrays (element i of thread t at
// [i * threads + t], conflict-free in shared memory): variables, the
// evaluated rate table, a snapshot of the variables for broadcast receivers,
// component locations and, when some location has several edges, the
// enabled-edge slot masks.
//
// Template options: SLOTS keeps the slot masks; LOC8 stores locations as
// 8-bit local indices (automata of at most 256 locations), otherwise as
// 16-bit global indices; GSTATE puts the state in per-CTA global slabs when
// it does not fit in shared memory.  The network layout comes from the
// kernel parameters, so pointers into the staged network are rebuilt from
// constants instead of occupying registers.
//
// The component order, the race tie-break, the Philox draws and every
// arithmetic step are those of the lane-group kernel and the CPU oracle
// (reference: simulation/simulation.cu:674-901).
#pragma once
#include "sim_common.cuh"

namespace csmc {
namespace detail {

// Delay of a component whose location is invariant-bounded, or whose rate
// is evaluated per component (uncommon; out of line).
static __device__ __noinline__ float slow_delay(const Net &n, VarView vars, VarView rates, uint32_t li, uint32_t x) {
    return comp_delay(n, vars, rates, li, x);
}

#ifndef CSMC_SERIAL_MIN_CTAS_PER_SM
#define CSMC_SERIAL_MIN_CTAS_PER_SM 5
#endif

template <bool LOC8>
struct LocStore {
    using T = uint16_t;  // global location index
};
template <>
struct LocStore<true> {
    using T = uint8_t;   // local location index
};

template <bool VERIFY, bool SLOTS, bool LOC8, bool GSTATE>
__global__ void __launch_bounds__(128, CSMC_SERIAL_MIN_CTAS_PER_SM) serial_kernel(const SimParams p) {
    using LocT = typename LocStore<LOC8>::T;
    extern __shared__ __align__(16) uint8_t smem[];
    stage_network(smem, p.blob, p.blob_bytes);
    __syncthreads();
    const Net n = net_view(smem, p.net);
    const uint32_t C = p.net.n_comps, V = p.net.n_vars, P = p.net.n_rate_prog;
    const uint32_t bits = ceil_log2(C);
    const bool rate_table = (p.net.flags & CSMC_NET_RATE_TABLE) && P > 0;

    // per-thread interleaved state
    const uint32_t T = blockDim.x, t = threadIdx.x;
    uint8_t *st = GSTATE ? p.state_global + static_cast<size_t>(blockIdx.x) * p.state_stride : smem + p.blob_bytes;
    float *fb = reinterpret_cast<float *>(st);
    const VarView vars{fb + t, T};
    const VarView rates{fb + V * T + t, T};
    const VarView shadow{fb + (V + P) * T + t, T};
    const uint32_t loc_bytes = LOC8 ? ((C * T + 3u) & ~3u) : ((2u * C * T + 3u) & ~3u);
    LocT *locs = reinterpret_cast<LocT *>(st + 4u * (2u * V + P) * T) + t;
    uint32_t *slotv = reinterpret_cast<uint32_t *>(st + 4u * (2u * V + P) * T + loc_bytes) + t;

    // global location index of component c in local location l / of its stored location
    auto global_of = [&](uint32_t c, uint32_t stored) -> uint32_t {
        return LOC8 ? n.comp[c].loc_begin + stored : stored;
    };
    auto store_of = [&](uint32_t c, uint32_t local) -> LocT {
        return static_cast<LocT>(LOC8 ? local : n.comp[c].loc_begin + local);
    };

    const uint32_t lane = threadIdx.x & 31u;
    const float T_end = p.horizon;
    const uint64_t cap = p.max_steps;
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
                // run initialisation (simulation.cu:766-831)
                for (uint32_t c = 0; c < C; ++c) {
                    locs[c * T] = store_of(c, n.comp[c].init_local);
                    if (SLOTS) slotv[c * T] = 0u;
                }
                for (uint32_t v = 0; v < V; ++v) vars[v] = n.var[v].init;
                double q0 = 0.0;
                if (p.var_id >= 0 && static_cast<uint32_t>(p.var_id) < V && n.var[p.var_id].kind == 0)
                    q0 = static_cast<double>(n.var[p.var_id].init);
                sc = RunScalars{q0, q0, 0xcbf29ce484222325ull, 0, -1, 0, 0};
                time = 0.0f;
                step = 0;
            }
        }

        // ---- end of run (simulation.cu:835-849, 887-893)
        const bool timeout = !(time < T_end);
        const bool at_goal = p.loc_mode && sc.goal;
        const bool at_cap = step >= cap;
        if (timeout || at_goal || at_cap) {
            const uint32_t flag_loc = (!timeout && at_goal) ? 1u : 0u;
            const uint32_t capped = (!timeout && !at_goal && at_cap) ? 1u : 0u;
            const double val = p.is_max ? sc.qmax : sc.qmin;
            uint32_t f = flag_loc;
            if (!p.loc_mode) f = p.is_max ? (val > p.threshold) : (val < p.threshold);
            if (p.flags) p.flags[ridx] = static_cast<uint8_t>(f);
            if (p.values) p.values[ridx] = val;
            if (p.steps) p.steps[ridx] = step;
            if (VERIFY) {
                if (p.digests) p.digests[ridx] = sc.digest;
                if (p.final_state) {
                    uint32_t *w = p.final_state + ridx * (C + V);
                    for (uint32_t c = 0; c < C; ++c) w[c] = global_of(c, locs[c * T]) - n.comp[c].loc_begin;
                    for (uint32_t v = 0; v < V; ++v) w[C + v] = f_bits(vars[v]);
                }
            }
            acc_hits += f;
            acc_steps += step;
            acc_capped += capped;
            have = false;
            continue;
        }

        // ---- broadcast receivers (SyncInSerial, simulation.cu:357-407):
        // enabled sets from the state the sender left (the snapshot), then
        // transitions in component order on the live state
        if (sc.chan > 0) {
            const int chan = sc.chan, sender = sc.sender;
            if (has_receivers(n, chan)) {
                for (uint32_t v = 0; v < V; ++v) shadow[v] = vars[v];
                for (uint32_t c = 0; c < C; ++c) {
                    if (static_cast<int>(c) == sender) continue;
                    const uint32_t li = global_of(c, locs[c * T]);
                    if (!n.loc[li].n_recv) continue;
                    const uint32_t m = recv_edges(n, shadow, li, chan);
                    if (!m) continue;
                    uint32_t sm = 0;
                    if (SLOTS) {
                        sm = write_slots(slotv[c * T], m);
                        slotv[c * T] = sm;
                    }
                    if (VERIFY) mix(sc.digest, c | 0x80000000u);
                    const uint32_t base = n.comp[c].loc_begin;
                    const uint32_t nl =
                        take_edge<VERIFY>(n, vars, sc, p.seed, p.var_id, run, step, c, li - base, m, sm, 1);
                    locs[c * T] = store_of(c, nl);
                }
            }
            sc.chan = 0;
            sc.sender = -1;
        }

        // ---- distinct rate programs, once per step
        if (rate_table)
            for (uint32_t j = 0; j < P; ++j) rates[j] = inv_rate(eval(n, vars, n.rate_prog[j]));

        // ---- delays and the race (simulation.cu:409-628)
        unsigned long long best = ~0ull;
        float bestd = 0.0f;
        for (uint32_t c = 0; c < C; c += 4) {
            const u32x4 blk = delay_block(p.seed, run, step, c >> 2);
#pragma unroll
            for (uint32_t k = 0; k < 4; ++k) {
                const uint32_t cc = c + k;
                if (cc < C) {
                    // fast path from the location's delay descriptor: the
                    // exponential delay with the literal 1/rate or the
                    // step's evaluated rate; zero-delay types and bounded
                    // locations take the general path
                    const uint32_t li = global_of(cc, locs[cc * T]);
                    const uint64_t dsc = n.loc_desc[li];
                    const uint32_t lo = static_cast<uint32_t>(dsc), fl = static_cast<uint32_t>(dsc >> 32);
                    const uint32_t x = word_of(blk, k);
                    float inv = __uint_as_float(lo);
                    if (fl & CSMC_DESC_PROG) inv = rates[lo];
                    float d = exp_delay(x, inv);
                    if (fl & (CSMC_DESC_ZERO | CSMC_DESC_INV | CSMC_DESC_EVAL))
                        d = (fl & CSMC_DESC_ZERO) ? 0.0f : slow_delay(n, vars, rates, li, x);
                    const unsigned long long key =
                        (static_cast<unsigned long long>(delay_key(d)) << 32) | bitrev_bits(cc, bits);
                    if (key < best) {
                        best = key;
                        bestd = d;
                    }
                }
            }
        }
        const uint32_t win = bitrev_bits(static_cast<uint32_t>(best & 0xffffffffull), bits);
        const float dmin = bestd;
        if (VERIFY) {
            mix(sc.digest, step);
            mix(sc.digest, win);
            mix(sc.digest, f_bits(dmin));
        }
        if (static_cast<double>(dmin) < kDblMax) {
            for (uint32_t j = 0; j < p.net.n_clocks; ++j) {  // simulation.cu:632-651
                const uint32_t v = n.clock[j];
                vars[v] = d2f(d_add(static_cast<double>(vars[v]), static_cast<double>(dmin)));
            }
            const uint32_t li = global_of(win, locs[win * T]);  // simulation.cu:656-667
            const uint32_t en = enabled_edges(n, vars, li);
            uint32_t sm = 0;
            if (SLOTS) {
                sm = write_slots(slotv[win * T], en);
                slotv[win * T] = sm;
            }
            if (en) {
                const uint32_t base = n.comp[win].loc_begin;
                const uint32_t nl =
                    take_edge<VERIFY>(n, vars, sc, p.seed, p.var_id, run, step, win, li - base, en, sm, 0);
                locs[win * T] = store_of(win, nl);
            } else if (VERIFY) {
                mix(sc.digest, 0xffffffffu);
            }
        }
        time = d2f(d_add(static_cast<double>(time), static_cast<double>(dmin)));  // simulation.cu:876-882
        ++step;
    }
    // lanes leave the loop at different times; aggregate per lane
    if (acc_hits) atomicAdd(p.scratch + 1, acc_hits);
    if (acc_steps) atomicAdd(p.scratch + 2, acc_steps);
    if (acc_capped) atomicAdd(p.scratch + 3, acc_capped);
}

}  // namespace detail

template <bool VERIFY, bool SLOTS, bool LOC8, bool GSTATE>
int serial_launch_one(const SimParams &p, int grid, int block, size_t smem, void *stream) {
    auto fn = detail::serial_kernel<VERIFY, SLOTS, LOC8, GSTATE>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool VERIFY, bool SLOTS, bool LOC8, bool GSTATE>
int serial_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::serial_kernel<VERIFY, SLOTS, LOC8, GSTATE>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
