// Lane-group simulation kernel (see sim.cuh for the mapping); instantiated
// per (lanes per run, components per lane) shape in sim_shapes_*.cu.
// Semantics follow the reference kernel line by line; file:line references
// are to simulation/simulation.cu of the reference.
#pragma once
#include "sim_common.cuh"

namespace csmc {
namespace detail {

struct RunState {  // per group, in shared memory (group_state_stride bytes)
    RunScalars sc;
    uint32_t pad2[2];
    float vars[1];  // n_vars entries, then n_rate_prog inverse rates, then
                    // (at group_vars_bytes) the slot masks [k * G + lane]
};

template <bool VERIFY>
static __device__ __noinline__ uint32_t group_take(const Net &n, RunState *s, uint64_t seed, int32_t var_id,
                                                   uint64_t run, uint32_t step, uint32_t c, uint32_t cur_loc,
                                                   uint32_t en, uint32_t slot_mask, uint32_t which) {
    return take_edge<VERIFY>(n, VarView{s->vars, 1}, s->sc, seed, var_id, run, step, c, cur_loc, en, slot_mask,
                             which);
}

// The winner's step (simulation.cu:656-667): enabled edges, slot update,
// transition.  Returns the new local location; *slots is updated.
template <bool VERIFY>
static __device__ __noinline__ uint32_t win_step(const Net &n, RunState *s, uint64_t seed, int32_t var_id,
                                                 uint64_t run, uint32_t step, uint32_t c, uint32_t cur_loc,
                                                 uint32_t *slots) {
    const uint32_t en = enabled_edges(n, VarView{s->vars, 1}, n.comp[c].loc_begin + cur_loc);
    *slots = write_slots(*slots, en);
    if (en) return group_take<VERIFY>(n, s, seed, var_id, run, step, c, cur_loc, en, *slots, 0);
    if (VERIFY) mix(s->sc.digest, 0xffffffffu);
    return cur_loc;
}

static __device__ __noinline__ uint32_t recv_mask(const Net &n, RunState *s, uint32_t li, int chan) {
    return recv_edges(n, VarView{s->vars, 1}, li, chan);
}

// One whole run (stream index `run`, output index `ridx`) simulated by the
// G lanes of a group: lane gl holds components gl*K .. gl*K+K-1 (C <= G*K)
// and their locations in registers; the group's scalars, variables, rate
// table and slot masks live in *s (slot masks are touched only by the
// step's winner and receivers, so they stay out of the registers).  Q supplies the
// query (seed, max_steps, threshold, horizon, var_id, loc_mode, is_max) and
// the per-run output arrays (flags, values, steps, digests, final_state; any
// may be null): the kernel parameters of one network, or one batch job.
// Lane 0 of the group writes the outputs and adds the run's hits, steps and
// capped flag to its accumulators.
template <int G, int K, bool VERIFY, class Q>
static __device__ __forceinline__ void group_run(const Net &n, RunState *s, const Q &q, uint64_t run,
                                                 uint64_t ridx, uint32_t gl,
                                                 uint32_t gbase, uint32_t gmask, unsigned long long &acc_hits,
                                                 unsigned long long &acc_steps, unsigned long long &acc_capped) {
    const uint32_t C = n.n_comps, V = n.n_vars;
    const uint32_t bits = ceil_log2(C);
    const bool rate_table = (n.flags & CSMC_NET_RATE_TABLE) && n.n_rate_prog > 0;
    const VarView vars{s->vars, 1};
    const VarView rates{s->vars + V, 1};
    const uint32_t c0 = gl * K;
    const float T = q.horizon;
    const uint64_t cap = q.max_steps;

    // run initialisation (simulation.cu:766-831)
    for (uint32_t v = gl; v < V; v += G) s->vars[v] = n.var[v].init;
    if (gl == 0) {
        double q0 = 0.0;
        if (q.var_id >= 0 && static_cast<uint32_t>(q.var_id) < V && n.var[q.var_id].kind == 0)
            q0 = static_cast<double>(n.var[q.var_id].init);
        s->sc.qmin = q0;
        s->sc.qmax = q0;
        s->sc.chan = 0;
        s->sc.sender = -1;
        s->sc.goal = 0;
        s->sc.digest = 0xcbf29ce484222325ull;
    }
    uint32_t loc[K];
    uint32_t *const slots =
        reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(s) + group_vars_bytes(V, n.n_rate_prog)) + gl;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const uint32_t c = c0 + k;
        loc[k] = c < C ? n.comp[c].loc_begin + n.comp[c].init_local : 0u;  // global location index
        slots[k * G] = 0u;
    }
    __syncwarp(gmask);

    float time = 0.0f;
    uint32_t step = 0;
    uint32_t flag = 0, capped = 0;
    while (time < T) {  // simulation.cu:835
        if (q.loc_mode && s->sc.goal) {  // simulation.cu:839-849
            flag = 1;
            break;
        }
        if (step >= cap) {
            capped = 1;
            break;
        }
        // ---- broadcast receivers (SyncInSerial, simulation.cu:357-407)
        const int chan = s->sc.chan;
        if (chan > 0) {
            const int sender = s->sc.sender;
            uint32_t rm[K];
            bool any = false;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                rm[k] = 0;
                const uint32_t c = c0 + k;
                if (c < C && static_cast<int>(c) != sender && n.loc[loc[k]].n_recv && has_receivers(n, chan)) {
                    rm[k] = recv_mask(n, s, loc[k], chan);
                    any |= rm[k] != 0;
                }
            }
            uint32_t pending = (__ballot_sync(gmask, any) & gmask) >> gbase;
            __syncwarp(gmask);  // every enabled set is taken before any receiver moves
            while (pending) {
                const uint32_t who = static_cast<uint32_t>(__ffs(pending) - 1);
                if (gl == who) {
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        if (!rm[k]) continue;
                        const uint32_t c = c0 + k;
                        const uint32_t base = n.comp[c].loc_begin;
                        const uint32_t sm = write_slots(slots[k * G], rm[k]);
                        slots[k * G] = sm;
                        if (VERIFY) mix(s->sc.digest, c | 0x80000000u);
                        loc[k] = base + group_take<VERIFY>(n, s, q.seed, q.var_id, run, step, c, loc[k] - base,
                                                           rm[k], sm, 1);
                    }
                }
                __syncwarp(gmask);
                pending &= pending - 1;
            }
            if (gl == 0) {
                s->sc.chan = 0;
                s->sc.sender = -1;
            }
            __syncwarp(gmask);
        }

        // ---- distinct rate programs, once per step per run
        if (rate_table) {
            for (uint32_t j = gl; j < n.n_rate_prog; j += G) rates[j] = inv_rate(eval(n, vars, n.rate_prog[j]));
            __syncwarp(gmask);
        }

        // ---- delays (simulation.cu:409-541)
        unsigned long long best = ~0ull;
        float bestd = 0.0f;
        u32x4 blk{0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint32_t c = c0 + k;
            if (c < C) {
                uint32_t x;
                if (K % 4 == 0) {
                    if (k % 4 == 0) blk = delay_block(q.seed, run, step, c >> 2);
                    x = word_of(blk, static_cast<uint32_t>(k & 3));
                } else {
                    x = delay_word(q.seed, run, step, c);
                }
                const float d = comp_delay(n, vars, rates, loc[k], x);
                const unsigned long long key =
                    (static_cast<unsigned long long>(delay_key(d)) << 32) | bitrev_bits(c, bits);
                if (key < best) {
                    best = key;
                    bestd = d;
                }
            }
        }
        // ---- race (simulation.cu:553-628): segmented butterfly min
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) {
            const unsigned long long ob = __shfl_xor_sync(gmask, best, off, G);
            const float od = __shfl_xor_sync(gmask, bestd, off, G);
            if (ob < best) {
                best = ob;
                bestd = od;
            }
        }
        const uint32_t win = bitrev_bits(static_cast<uint32_t>(best & 0xffffffffull), bits);
        const float dmin = bestd;
        const uint32_t owner = win / K;
        if (VERIFY && gl == owner) {
            mix(s->sc.digest, step);
            mix(s->sc.digest, win);
            mix(s->sc.digest, f_bits(dmin));
        }
        if (static_cast<double>(dmin) < kDblMax) {
            // clocks advance (simulation.cu:632-651)
            for (uint32_t j = gl; j < n.n_clocks; j += G) {
                const uint32_t v = n.clock[j];
                s->vars[v] = d2f(d_add(static_cast<double>(s->vars[v]), static_cast<double>(dmin)));
            }
            __syncwarp(gmask);
            if (gl == owner) {
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    if (c0 + k != win) continue;
                    const uint32_t base = n.comp[win].loc_begin;
                    loc[k] = base + win_step<VERIFY>(n, s, q.seed, q.var_id, run, step, win, loc[k] - base,
                                                     &slots[k * G]);
                }
            }
            __syncwarp(gmask);
        }
        time = d2f(d_add(static_cast<double>(time), static_cast<double>(dmin)));  // simulation.cu:876-882
        ++step;
    }

    // per-run outputs (simulation.cu:887-893)
    if (gl == 0) {
        const double val = q.is_max ? s->sc.qmax : s->sc.qmin;
        uint32_t f = flag;
        if (!q.loc_mode) f = q.is_max ? (val > q.threshold) : (val < q.threshold);
        if (q.flags) q.flags[ridx] = static_cast<uint8_t>(f);
        if (q.values) q.values[ridx] = val;
        if (q.steps) q.steps[ridx] = step;
        if (VERIFY && q.digests) q.digests[ridx] = s->sc.digest;
        acc_hits += f;
        acc_steps += step;
        acc_capped += capped;
    }
    if (VERIFY && q.final_state) {
        uint32_t *w = q.final_state + ridx * (C + V);
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (c0 + k < C) w[c0 + k] = loc[k] - n.comp[c0 + k].loc_begin;
        for (uint32_t v = gl; v < V; v += G) w[C + v] = f_bits(s->vars[v]);
    }
    __syncwarp(gmask);
}

#ifndef CSMC_MIN_CTAS_PER_SM
#define CSMC_MIN_CTAS_PER_SM 2
#endif

template <int G, int K, bool VERIFY>
__global__ void __launch_bounds__(256, CSMC_MIN_CTAS_PER_SM) sim_kernel(const SimParams p) {
    extern __shared__ __align__(16) uint8_t smem[];
    stage_network(smem, p.blob, p.blob_bytes);
    __syncthreads();
    const Net n = net_view(smem);

    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gl = lane % G;  // lane within group
    const uint32_t gbase = lane - gl;
    const uint32_t gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << gbase);
    RunState *s = reinterpret_cast<RunState *>(smem + p.blob_bytes + (threadIdx.x / G) * p.state_stride);

    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;
    for (;;) {
        unsigned long long ridx = 0;
        if (gl == 0) ridx = atomicAdd(p.scratch, 1ull);
        ridx = __shfl_sync(gmask, ridx, 0, G);
        if (ridx >= p.n_runs) break;
        group_run<G, K, VERIFY>(n, s, p, p.first_run + ridx, ridx, gl, gbase, gmask, acc_hits, acc_steps,
                                acc_capped);
    }
    if (gl == 0) {
        if (acc_hits) atomicAdd(p.scratch + 1, acc_hits);
        if (acc_steps) atomicAdd(p.scratch + 2, acc_steps);
        if (acc_capped) atomicAdd(p.scratch + 3, acc_capped);
    }
}

}  // namespace detail

template <int G, int K, bool VERIFY>
int launch_one(const SimParams &p, int grid, int block, size_t smem, void *stream) {
    auto fn = detail::sim_kernel<G, K, VERIFY>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <int G, int K, bool VERIFY>
int occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::sim_kernel<G, K, VERIFY>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

// Explicit instantiation of the launch helpers for one shape.
#define CSMC_INSTANTIATE_SHAPE(GG, KK)                                                  \
    template int launch_one<GG, KK, false>(const SimParams &, int, int, size_t, void *); \
    template int launch_one<GG, KK, true>(const SimParams &, int, int, size_t, void *);  \
    template int occupancy_one<GG, KK, false>(int, size_t, int *);                        \
    template int occupancy_one<GG, KK, true>(int, size_t, int *);

}  // namespace csmc
