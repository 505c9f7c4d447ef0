// Importance-sampling simulation: the thread-per-run kernel with every
// exponential delay drawn under the proposal network's tilt (csmc_mlp.h),
// the path's log-likelihood ratio carried in FP64, and a replay mode that
// writes the CE training rows of listed runs.
//
// Per step and run, the proposal needs theta for each location class (local
// location index modulo 4): the four rows are evaluated on CUDA cores from
// FP32 copies of the BF16 weights in shared memory, with the operation order
// of mlp_theta, so runs are bit-identical to the CPU oracle's.  Replay mode
// writes exactly four rows per step of each listed run at a caller-given
// offset (rows of classes without a tilted component, and of steps in which
// nothing can fire, are zero-weighted), so the row set does not depend on
// scheduling.
#pragma once
#include "../include/csmc_mlp.h"
#include "sim_run.cuh"

namespace csmc {
namespace detail {

struct MlpSmem {  // FP32 copies of the proposal network
    float w1[CSMC_MLP_HID][CSMC_MLP_IN];
    float w2[CSMC_MLP_HID][CSMC_MLP_HID];
    float b1[CSMC_MLP_HID], b2[CSMC_MLP_HID], w3[CSMC_MLP_HID];
    float b3, pad[3];
};

static __device__ __forceinline__ void stage_mlp(MlpSmem *m, const MlpParams *P) {
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID * CSMC_MLP_IN; i += blockDim.x)
        (&m->w1[0][0])[i] = bf16_to_f((&P->w1[0][0])[i]);
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID * CSMC_MLP_HID; i += blockDim.x)
        (&m->w2[0][0])[i] = bf16_to_f((&P->w2[0][0])[i]);
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID; i += blockDim.x) {
        m->b1[i] = P->b1[i];
        m->b2[i] = P->b2[i];
        m->w3[i] = P->w3[i];
    }
    if (threadIdx.x == 0) m->b3 = P->b3;
}

// theta of one feature row; the operations of mlp_theta in the same order
static __device__ __noinline__ float mlp_theta_smem(const MlpSmem *m, const float *x) {
    float h1[CSMC_MLP_HID];
#pragma unroll
    for (int j = 0; j < CSMC_MLP_HID; ++j) {
        float z = m->b1[j];
#pragma unroll
        for (int i = 0; i < CSMC_MLP_IN; ++i) z = f_fma(x[i], m->w1[j][i], z);
        h1[j] = bf16_round(gelu_f(z));
    }
    float th = m->b3;
    for (int k = 0; k < CSMC_MLP_HID; ++k) {
        float z = m->b2[k];
#pragma unroll
        for (int j = 0; j < CSMC_MLP_HID; ++j) z = f_fma(h1[j], m->w2[k][j], z);
        th = f_fma(gelu_f(z), m->w3[k], th);
    }
    return th < -CSMC_MLP_THETA_MAX ? -CSMC_MLP_THETA_MAX : (th > CSMC_MLP_THETA_MAX ? CSMC_MLP_THETA_MAX : th);
}

// Delay of a component on the general path under the proposal.
static __device__ __noinline__ float is_slow_delay(const Net &n, VarView vars, VarView rates, uint32_t li, uint32_t x,
                                                   float mfac, bool *tilted, float *inv_o, float *invp_o) {
    *tilted = false;
    *inv_o = *invp_o = 0.0f;
    const csmc_loc L = n.loc[li];
    if (L.type > 1) return 0.0f;
    if (L.n_inv) {
        double max_delay;
        if (delay_bound(n, vars, L, max_delay)) return uniform_delay(x, max_delay);
    }
    float inv;
    if (n.flags & CSMC_NET_RATE_TABLE) {
        const uint32_t slot = n.loc_rate[li];
        inv = (slot & CSMC_RATE_PROG_BIT) ? rates[slot & ~CSMC_RATE_PROG_BIT] : n.inv_lit[slot];
    } else {
        inv = inv_rate(eval(n, vars, L.rate));
    }
    float invp = inv;
    if (tiltable(inv)) {
        invp = f_mul(inv, mfac);
        *tilted = true;
    }
    *inv_o = inv;
    *invp_o = invp;
    return exp_delay(x, invp);
}

#ifndef CSMC_IS_MIN_CTAS_PER_SM
#define CSMC_IS_MIN_CTAS_PER_SM 2
#endif

template <bool TRACE, bool SLOTS, bool LOC8>
__global__ void __launch_bounds__(128, CSMC_IS_MIN_CTAS_PER_SM) is_kernel(const IsParams ip) {
    const SimParams &p = ip.s;
    extern __shared__ __align__(16) uint8_t smem[];
    stage_network(smem, p.blob, p.blob_bytes);
    MlpSmem *mlp = reinterpret_cast<MlpSmem *>(smem + p.blob_bytes);
    stage_mlp(mlp, ip.mlp);
    __syncthreads();
    const Net n = net_view(smem, p.net);
    const uint32_t C = p.net.n_comps, V = p.net.n_vars, P = p.net.n_rate_prog;
    const bool rate_table = (p.net.flags & CSMC_NET_RATE_TABLE) && P > 0;
    const uint32_t bits = ceil_log2(C);
    const uint32_t n_int = V < 4 ? V : 4;

    const uint32_t T = blockDim.x, t = threadIdx.x;
    uint8_t *st = smem + p.blob_bytes + sizeof(MlpSmem);
    const RunView<LOC8> rv = carve_run_view<LOC8>(st, V, P, C, T, t);

    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;
    bool have = false;
    unsigned long long ridx = 0;
    uint64_t run = 0;
    float time = 0.0f;
    uint32_t step = 0;
    double logw = 0.0;
    RunScalars sc{0.0, 0.0, 0, 0, -1, 0, 0};
    MlpRow *rows = nullptr;
    float row_w = 0.0f;

    for (;;) {
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
                if (TRACE) {
                    run = p.first_run + ip.trace_runs[ridx];
                    row_w = ip.trace_w[ridx];
                    rows = ip.rows + ip.row_offset[ridx];
                } else {
                    run = p.first_run + ridx;
                }
                run_init<SLOTS, LOC8>(n, C, V, rv, sc, p.var_id);
                time = 0.0f;
                step = 0;
                logw = 0.0;
            }
        }

        const RunEnd e = run_end(sc, time, p.horizon, step, p.max_steps, p.loc_mode, p.is_max, p.threshold);
        if (e.done) {
            if (!TRACE) {
                if (p.flags) p.flags[ridx] = static_cast<uint8_t>(e.flag);
                if (p.values) p.values[ridx] = e.value;
                if (p.steps) p.steps[ridx] = step;
                if (ip.logw) ip.logw[ridx] = logw;
                if (ip.wvals) ip.wvals[ridx] = e.flag ? exp2_d(d_mul(logw, 1.4426950408889634)) : 0.0;
            }
            acc_hits += e.flag;
            acc_steps += step;
            acc_capped += e.capped;
            have = false;
            continue;
        }

        run_receivers<false, SLOTS, LOC8>(n, C, V, rv, sc, p.seed, p.var_id, run, step);
        if (rate_table)
            for (uint32_t j = 0; j < P; ++j) rv.rates[j] = inv_rate(eval(n, rv.vars, n.rate_prog[j]));

        // ---- the proposal's factor per location class
        float v4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (uint32_t i = 0; i < n_int; ++i) v4[i] = rv.vars[i];
        float mfac[CSMC_MLP_CLASSES];
        float feat[CSMC_MLP_IN];
#pragma unroll
        for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) {
            mlp_features(l, v4, n_int, C, time, p.horizon, feat);
            mfac[l] = tilt_factor(mlp_theta_smem(mlp, feat));
        }

        // ---- delays and the race under the proposal
        unsigned long long best = ~0ull;
        float bestd = 0.0f, best_inv = 0.0f, best_invp = 0.0f;
        bool best_tilted = false;
        double rate_sum = 0.0;
        double inv_sum[CSMC_MLP_CLASSES] = {0.0, 0.0, 0.0, 0.0};
        uint32_t cls_count = 0;  // 8 bits per class (saturating flag use only)
        for (uint32_t c = 0; c < C; c += 4) {
            const u32x4 blk = delay_block(p.seed, run, step, c >> 2);
#pragma unroll
            for (uint32_t k = 0; k < 4; ++k) {
                const uint32_t cc = c + k;
                if (cc < C) {
                    const uint32_t li = rv.loc(n, cc);
                    const uint32_t l = (li - n.comp[cc].loc_begin) & 3u;
                    const uint64_t dsc = n.loc_desc[li];
                    const uint32_t lo = static_cast<uint32_t>(dsc), fl = static_cast<uint32_t>(dsc >> 32);
                    const uint32_t x = word_of(blk, k);
                    const float m = l == 0 ? mfac[0] : (l == 1 ? mfac[1] : (l == 2 ? mfac[2] : mfac[3]));
                    float d, inv = 0.0f, invp = 0.0f;
                    bool tilted = false;
                    if (fl & (CSMC_DESC_ZERO | CSMC_DESC_INV | CSMC_DESC_EVAL)) {
                        if (fl & CSMC_DESC_ZERO) d = 0.0f;
                        else d = is_slow_delay(n, rv.vars, rv.rates, li, x, m, &tilted, &inv, &invp);
                    } else {
                        inv = __uint_as_float(lo);
                        if (fl & CSMC_DESC_PROG) inv = rv.rates[lo];
                        invp = inv;
                        if (tiltable(inv)) {
                            invp = f_mul(inv, m);
                            tilted = true;
                        }
                        d = exp_delay(x, invp);
                    }
                    if (tilted) {
                        rate_sum = d_add(rate_sum, rate_change(inv, invp));
                        if (TRACE) {
                            const double r = d_div(1.0, static_cast<double>(inv));
                            if (l == 0) inv_sum[0] = d_add(inv_sum[0], r);
                            else if (l == 1) inv_sum[1] = d_add(inv_sum[1], r);
                            else if (l == 2) inv_sum[2] = d_add(inv_sum[2], r);
                            else inv_sum[3] = d_add(inv_sum[3], r);
                            cls_count |= 1u << (8 * l);
                        }
                    }
                    const unsigned long long key =
                        (static_cast<unsigned long long>(delay_key(d)) << 32) | bitrev_bits(cc, bits);
                    if (key < best) {
                        best = key;
                        bestd = d;
                        best_inv = inv;
                        best_invp = invp;
                        best_tilted = tilted;
                    }
                }
            }
        }
        const uint32_t win = bitrev_bits(static_cast<uint32_t>(best & 0xffffffffull), bits);
        const bool finite = static_cast<double>(bestd) < kDblMax;
        if (finite) logw = d_add(logw, step_log_ratio(rate_sum, bestd, best_tilted, best_inv, best_invp));
        if (TRACE) {
            const uint32_t wl = (rv.loc(n, win) - n.comp[win].loc_begin) & 3u;
#pragma unroll
            for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) {
                mlp_features(l, v4, n_int, C, time, p.horizon, feat);
                MlpRow r;
#pragma unroll
                for (int i = 0; i < CSMC_MLP_IN; ++i) r.x[i] = f_to_bf16(feat[i]);
                const bool has = finite && ((cls_count >> (8 * l)) & 1u);
                const double s = l == 0 ? inv_sum[0] : (l == 1 ? inv_sum[1] : (l == 2 ? inv_sum[2] : inv_sum[3]));
                r.a = has ? row_a(s, bestd, row_w) : 0.0f;
                r.b = (has && best_tilted && wl == l) ? row_w : 0.0f;
                rows[4 * step + l] = r;
            }
        }
        run_commit<false, SLOTS, LOC8>(n, p.net.n_clocks, rv, sc, p.seed, p.var_id, run, step, time, win, bestd);
    }
    if (acc_hits) atomicAdd(p.scratch + 1, acc_hits);
    if (acc_steps) atomicAdd(p.scratch + 2, acc_steps);
    if (acc_capped) atomicAdd(p.scratch + 3, acc_capped);
}

}  // namespace detail

template <bool TRACE, bool SLOTS, bool LOC8>
int is_launch_one(const IsParams &p, int grid, int block, size_t smem, void *stream) {
    auto fn = detail::is_kernel<TRACE, SLOTS, LOC8>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool TRACE, bool SLOTS, bool LOC8>
int is_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::is_kernel<TRACE, SLOTS, LOC8>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
