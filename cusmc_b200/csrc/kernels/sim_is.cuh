// Importance-sampling simulation: one warp per run, every exponential delay
// drawn under the proposal network's tilt (csmc_mlp.h), the path's
// log-likelihood ratio carried in FP64, and a replay mode that writes the CE
// training rows of listed runs.
//
// A warp takes a run from the global counter and steps it to its end:
//   * lane 0 owns the run's scalars (query extremes, pending broadcast) and
//     does the serial parts, the broadcast receivers and the winner's
//     transition, on the run state in the warp's shared-memory slab (the
//     thread-per-run layout of sim_run.cuh with one thread);
//   * the rate table is evaluated across the lanes;
//   * theta of the four location classes (local location index modulo 4)
//     comes either from CUDA cores, lane L computing hidden units L and
//     L + 32 of the four feature rows in the operation order of mlp_theta
//     (bit-identical to the CPU oracle), or from warp-level BF16 MMAs
//     (mma.sync m16n8k16, FP32 accumulation) on one 16-row tile whose rows
//     0..3 are the classes; it is evaluated only when the step's features
//     differ from those of the warp's previous evaluation (theta depends on
//     nothing else), which skips most steps that change no variable;
//   * the race: lane L draws the Philox blocks q = L, L + 32, ...
//     (components 4q .. 4q + 3), keeps its smallest (delay key, bit-reversed
//     index) and its partial sums, and butterflies give the winner and the
//     sums in the warp order of csmc_mlp.h (warp_lane_of, warp_tree_d).
// A run advances one step per warp-step, so a launch of a few thousand runs
// (a CE round, the replay of its elite runs) takes about as long as its
// longest run at warp speed rather than at thread speed.
// Weights and estimates are exact for whichever theta a run used: the
// log-likelihood ratio is computed from the rates the run was drawn with.
// Replay mode writes exactly four rows per step of each listed run at a
// caller-given offset (rows of classes without a tilted component, and of
// steps in which nothing can fire, are zero-weighted), so the row set does
// not depend on scheduling; replay uses the evaluation the runs were drawn
// with, so it follows the same paths.
#pragma once
#include "../include/csmc_mlp.h"
#include "sim_run.cuh"

#ifndef CSMC_IS_MIN_CTAS_PER_SM
#define CSMC_IS_MIN_CTAS_PER_SM 2
#endif

namespace csmc {
namespace detail {

constexpr unsigned kFullWarp = 0xffffffffu;

struct MlpSmem {  // the proposal network in shared memory
    float w1t[CSMC_MLP_IN][CSMC_MLP_HID];   // FP32 copies of the BF16 weights, [input][unit]
    float w2t[CSMC_MLP_HID][CSMC_MLP_HID];  // [input unit][output unit]
    float b1[CSMC_MLP_HID], b2[CSMC_MLP_HID], w3[CSMC_MLP_HID];
    float b3, pad[3];
    uint16_t w1h[CSMC_MLP_HID][CSMC_MLP_IN];  // BF16, [unit][input]: MMA B fragments
    uint16_t w2h[CSMC_MLP_HID][CSMC_MLP_HID];
};
static_assert(sizeof(MlpSmem) % 16 == 0, "warp slabs follow the proposal network 16-byte aligned");

static __device__ __forceinline__ void stage_mlp(MlpSmem *m, const MlpParams *P) {
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID * CSMC_MLP_IN; i += blockDim.x) {
        const uint16_t w = (&P->w1[0][0])[i];
        (&m->w1h[0][0])[i] = w;
        m->w1t[i % CSMC_MLP_IN][i / CSMC_MLP_IN] = bf16_to_f(w);
    }
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID * CSMC_MLP_HID; i += blockDim.x) {
        const uint16_t w = (&P->w2[0][0])[i];
        (&m->w2h[0][0])[i] = w;
        m->w2t[i % CSMC_MLP_HID][i / CSMC_MLP_HID] = bf16_to_f(w);
    }
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID; i += blockDim.x) {
        m->b1[i] = P->b1[i];
        m->b2[i] = P->b2[i];
        m->w3[i] = P->w3[i];
    }
    if (threadIdx.x == 0) m->b3 = P->b3;
}

// Input i of class r's feature row: the class one-hot, then the run's
// shared features x[4..15] (mlp_features).
static __device__ __forceinline__ float feat_of(const float *x, uint32_t r, int i) {
    return i < 4 ? (static_cast<uint32_t>(i) == r ? 1.0f : 0.0f) : x[i];
}

// ---- theta on CUDA cores: the operations of mlp_theta ----------------------
// h1s: the warp's [64 units][4 rows] staging of the first hidden layer.
static __device__ __forceinline__ void theta_exact(const MlpSmem *m, float *h1s, const float *x,
                                                   float (&theta)[CSMC_MLP_CLASSES]) {
    const uint32_t lane = threadIdx.x & 31u;
    float za[4], zb[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        za[r] = m->b1[lane];
        zb[r] = m->b1[lane + 32];
    }
#pragma unroll
    for (int i = 0; i < CSMC_MLP_IN; ++i) {
        const float wa = m->w1t[i][lane], wb = m->w1t[i][lane + 32];
#pragma unroll
        for (uint32_t r = 0; r < 4; ++r) {
            const float xi = feat_of(x, r, i);
            za[r] = f_fma(xi, wa, za[r]);
            zb[r] = f_fma(xi, wb, zb[r]);
        }
    }
    __syncwarp();  // the previous step's readers of h1s are done
    float4 *h4 = reinterpret_cast<float4 *>(h1s);
    h4[lane] = make_float4(bf16_round(gelu_f(za[0])), bf16_round(gelu_f(za[1])), bf16_round(gelu_f(za[2])),
                           bf16_round(gelu_f(za[3])));
    h4[lane + 32] = make_float4(bf16_round(gelu_f(zb[0])), bf16_round(gelu_f(zb[1])), bf16_round(gelu_f(zb[2])),
                                bf16_round(gelu_f(zb[3])));
    __syncwarp();
    float ya[4], yb[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        ya[r] = m->b2[lane];
        yb[r] = m->b2[lane + 32];
    }
#pragma unroll 8
    for (int j = 0; j < CSMC_MLP_HID; ++j) {
        const float4 h = h4[j];
        const float wa = m->w2t[j][lane], wb = m->w2t[j][lane + 32];
        ya[0] = f_fma(h.x, wa, ya[0]);
        ya[1] = f_fma(h.y, wa, ya[1]);
        ya[2] = f_fma(h.z, wa, ya[2]);
        ya[3] = f_fma(h.w, wa, ya[3]);
        yb[0] = f_fma(h.x, wb, yb[0]);
        yb[1] = f_fma(h.y, wb, yb[1]);
        yb[2] = f_fma(h.z, wb, yb[2]);
        yb[3] = f_fma(h.w, wb, yb[3]);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        float s = f_fma(gelu_f(yb[r]), m->w3[lane + 32], f_fma(gelu_f(ya[r]), m->w3[lane], 0.0f));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s = f_add(s, __shfl_xor_sync(kFullWarp, s, off));
        theta[r] = clip_theta(f_add(m->b3, s));
    }
}

// ---- theta on tensor cores ---------------------------------------------------

static __device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    return static_cast<uint32_t>(f_to_bf16(lo)) | (static_cast<uint32_t>(f_to_bf16(hi)) << 16);
}

// D += A . B, A 16x16 (row), B 16x8 (col), BF16 operands, FP32 accumulators
static __device__ __forceinline__ void mma_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                 uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// GELU (tanh form) with the library exponential and reciprocal
static __device__ __forceinline__ float gelu_tc(float x) {
    const float s = gelu_arg(x);
    return x * __frcp_rn(1.0f + exp2f(-1.44269502f * s));
}

static __device__ __forceinline__ uint32_t ld_u32(const uint16_t *p) { return *reinterpret_cast<const uint32_t *>(p); }

// The four classes' theta from one m16 tile: lane (g, tig) = (lane / 4,
// lane % 4) holds row g's A-fragment words; rows 4..15 are zero.  The first
// layer's accumulators become the second layer's A fragments in registers
// (output n-tile 2q is K step q's low half, 2q + 1 its high half).
static __device__ __forceinline__ void theta_tc(const MlpSmem *m, const float *x, float (&theta)[CSMC_MLP_CLASSES]) {
    const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, tig = lane & 3u;
    const uint32_t onehot = pack_bf16(g == 2 * tig ? 1.0f : 0.0f, g == 2 * tig + 1 ? 1.0f : 0.0f);
    const uint32_t p2 = pack_bf16(x[4], x[5]), p3 = pack_bf16(x[6], x[7]);
    const uint32_t p4 = pack_bf16(x[8], x[9]), p5 = pack_bf16(x[10], x[11]);
    const uint32_t p6 = pack_bf16(x[12], x[13]), p7 = pack_bf16(x[14], x[15]);
    uint32_t a0 = tig < 2 ? onehot : (tig == 2 ? p2 : p3);                  // inputs 2 tig, 2 tig + 1
    uint32_t a2 = tig == 0 ? p4 : (tig == 1 ? p5 : (tig == 2 ? p6 : p7));  // inputs 2 tig + 8, + 9
    if (g >= CSMC_MLP_CLASSES) a0 = a2 = 0u;
    uint32_t hA[4][2];
#pragma unroll
    for (uint32_t nt = 0; nt < 8; ++nt) {
        const uint16_t *wr = &m->w1h[8 * nt + g][0];
        float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        mma_16816(d, a0, 0u, a2, 0u, ld_u32(wr + 2 * tig), ld_u32(wr + 2 * tig + 8));
        const uint32_t col = 8 * nt + 2 * tig;
        hA[nt >> 1][nt & 1] = pack_bf16(gelu_tc(d[0] + m->b1[col]), gelu_tc(d[1] + m->b1[col + 1]));
    }
    float s = 0.0f;
#pragma unroll
    for (uint32_t nt = 0; nt < 8; ++nt) {
        float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            const uint16_t *wr = &m->w2h[8 * nt + g][16 * q];
            mma_16816(d, hA[q][0], 0u, hA[q][1], 0u, ld_u32(wr + 2 * tig), ld_u32(wr + 2 * tig + 8));
        }
        const uint32_t col = 8 * nt + 2 * tig;
        s = fmaf(gelu_tc(d[0] + m->b2[col]), m->w3[col], s);
        s = fmaf(gelu_tc(d[1] + m->b2[col + 1]), m->w3[col + 1], s);
    }
    s += __shfl_xor_sync(kFullWarp, s, 1);
    s += __shfl_xor_sync(kFullWarp, s, 2);
    const float th = clip_theta(m->b3 + s);  // row g in lanes 4g .. 4g + 3
#pragma unroll
    for (uint32_t r = 0; r < CSMC_MLP_CLASSES; ++r) theta[r] = __shfl_sync(kFullWarp, th, 4 * r);
}

// ---- the race under the proposal ------------------------------------------

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

struct LaneRace {  // one lane's share of a step's race
    unsigned long long best;
    float bestd, best_inv, best_invp;
    bool best_tilted;
    double rate_sum;                   // this lane's sum of 1/inv' - 1/inv over tilted components
    double inv_sum[CSMC_MLP_CLASSES];  // replay: per class, this lane's sum of 1/inv of tilted components
    uint32_t cls_present;              // replay: bit l: this lane has a tilted component of class l
};

template <bool TRACE, bool LOC8>
static __device__ __forceinline__ void lane_race(const Net &n, uint32_t C, uint32_t bits, const RunView<LOC8> &rv,
                                                 uint64_t seed, uint64_t run, uint32_t step,
                                                 const float (&mfac)[CSMC_MLP_CLASSES], LaneRace &R) {
    const uint32_t lane = threadIdx.x & 31u;
    R.best = ~0ull;
    R.bestd = R.best_inv = R.best_invp = 0.0f;
    R.best_tilted = false;
    R.rate_sum = 0.0;
#pragma unroll
    for (int l = 0; l < CSMC_MLP_CLASSES; ++l) R.inv_sum[l] = 0.0;
    R.cls_present = 0;
    // Per class, the last tilted 1/rate seen and its two FP64 quotients: the
    // class's factor is fixed for the step, so equal 1/rate gives equal bits
    // and the divisions run once per distinct (class, 1/rate) pair.
    float k_inv[CSMC_MLP_CLASSES] = {-1.0f, -1.0f, -1.0f, -1.0f};
    double k_diff[CSMC_MLP_CLASSES] = {0.0, 0.0, 0.0, 0.0};
    double k_rec[CSMC_MLP_CLASSES] = {0.0, 0.0, 0.0, 0.0};
    for (uint32_t q = lane; 4u * q < C; q += 32u) {
        const u32x4 blk = delay_block(seed, run, step, q);
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t cc = 4u * q + k;
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
                    const float kv = l == 0 ? k_inv[0] : (l == 1 ? k_inv[1] : (l == 2 ? k_inv[2] : k_inv[3]));
                    double diff, r = 0.0;
                    if (kv == inv) {
                        diff = l == 0 ? k_diff[0] : (l == 1 ? k_diff[1] : (l == 2 ? k_diff[2] : k_diff[3]));
                        if (TRACE) r = l == 0 ? k_rec[0] : (l == 1 ? k_rec[1] : (l == 2 ? k_rec[2] : k_rec[3]));
                    } else {
                        diff = rate_change(inv, invp);
                        if (TRACE) r = d_div(1.0, static_cast<double>(inv));
#pragma unroll
                        for (int j = 0; j < CSMC_MLP_CLASSES; ++j)
                            if (static_cast<uint32_t>(j) == l) {
                                k_inv[j] = inv;
                                k_diff[j] = diff;
                                k_rec[j] = r;
                            }
                    }
                    R.rate_sum = d_add(R.rate_sum, diff);
                    if (TRACE) {
                        if (l == 0) R.inv_sum[0] = d_add(R.inv_sum[0], r);
                        else if (l == 1) R.inv_sum[1] = d_add(R.inv_sum[1], r);
                        else if (l == 2) R.inv_sum[2] = d_add(R.inv_sum[2], r);
                        else R.inv_sum[3] = d_add(R.inv_sum[3], r);
                        R.cls_present |= 1u << l;
                    }
                }
                const unsigned long long key =
                    (static_cast<unsigned long long>(delay_key(d)) << 32) | bitrev_bits(cc, bits);
                if (key < R.best) {
                    R.best = key;
                    R.bestd = d;
                    R.best_inv = inv;
                    R.best_invp = invp;
                    R.best_tilted = tilted;
                }
            }
        }
    }
}

// The butterfly of warp_tree_d: lane L adds lane L ^ off's value to its own.
static __device__ __forceinline__ double warp_sum_d(double s) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s = d_add(s, __shfl_xor_sync(kFullWarp, s, off));
    return s;
}

// ---- the kernel ----------------------------------------------------------------
template <bool TC, bool TRACE, bool SLOTS, bool LOC8>
__global__ void __launch_bounds__(CSMC_IS_BLOCK, CSMC_IS_MIN_CTAS_PER_SM) is_warp_kernel(const IsParams ip) {
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
    const uint32_t lane = threadIdx.x & 31u;
    uint8_t *slab = smem + p.blob_bytes + sizeof(MlpSmem) + static_cast<size_t>(threadIdx.x >> 5) * ip.slab_bytes;
    float *h1s = reinterpret_cast<float *>(slab);
    const RunView<LOC8> rv =
        carve_run_view<LOC8>(slab + (TC ? 0u : 4u * CSMC_MLP_HID * CSMC_MLP_CLASSES), V, P, C, 1, 0);

    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;
    RunScalars sc{0.0, 0.0, 0, 0, -1, 0, 0};  // lane 0's copy is the run's
    // theta is a function of the shared features x[4..15] alone (the network
    // is fixed for the launch): the last evaluated features and their class
    // factors, kept across steps and runs (steps that change no variable
    // and stay within one 1/64 step of t / T reuse them)
    uint32_t x_last[CSMC_MLP_IN - 4];
#pragma unroll
    for (int i = 0; i < CSMC_MLP_IN - 4; ++i) x_last[i] = 0xffffffffu;  // a NaN: never equal to a feature
    float mfac[CSMC_MLP_CLASSES] = {1.0f, 1.0f, 1.0f, 1.0f};
    // the last tilted winner's 1/rate and 1/rate' bits and its log term
    uint32_t w_inv = 0xffffffffu, w_invp = 0xffffffffu;
    double w_term = 0.0;

    for (;;) {
        unsigned long long ridx = 0;
        if (lane == 0) ridx = atomicAdd(p.scratch, 1ull);
        ridx = __shfl_sync(kFullWarp, ridx, 0);
        if (ridx >= p.n_runs) break;
        uint64_t run;
        float row_w = 0.0f;
        uint64_t row0 = 0;  // replay: the run's first row in the buffer
        if (TRACE) {
            run = p.first_run + ip.trace_runs[ridx];
            row_w = ip.trace_w[ridx];
            row0 = ip.row_offset[ridx];
        } else {
            run = p.first_run + ridx;
        }

        // run initialisation (run_init, across the lanes)
        for (uint32_t c = lane; c < C; c += 32u) {
            rv.set_local(n, c, n.comp[c].init_local);
            if (SLOTS) rv.slotv[c] = 0u;
        }
        for (uint32_t v = lane; v < V; v += 32u) rv.vars[v] = n.var[v].init;
        if (lane == 0) {
            double q0 = 0.0;
            if (p.var_id >= 0 && static_cast<uint32_t>(p.var_id) < V && n.var[p.var_id].kind == 0)
                q0 = static_cast<double>(n.var[p.var_id].init);
            sc = RunScalars{q0, q0, 0xcbf29ce484222325ull, 0, -1, 0, 0};
        }
        __syncwarp();

        float time = 0.0f;
        uint32_t step = 0;
        double logw = 0.0;
        // the rate table is a function of the variables: evaluated on a
        // run's first step and after steps that can have changed a variable
        // (a transition, a receiver, or clocks advancing)
        bool stale = true;
        for (;;) {
            int done = 0;
            if (lane == 0) {
                const RunEnd e = run_end(sc, time, p.horizon, step, p.max_steps, p.loc_mode, p.is_max, p.threshold);
                done = e.done;
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
                }
            }
            if (__shfl_sync(kFullWarp, done, 0)) break;

            // pending broadcast receivers (serial, lane 0), then the rate table
            int moved = 0;
            if (lane == 0) moved = run_receivers<false, SLOTS>(n, C, V, rv, sc, p.seed, p.var_id, run, step);
            __syncwarp();
            stale = stale || __shfl_sync(kFullWarp, moved, 0) != 0;
            if (rate_table && stale) {
                for (uint32_t j = lane; j < P; j += 32u) rv.rates[j] = inv_rate(eval(n, rv.vars, n.rate_prog[j]));
                __syncwarp();
            }

            // the proposal's class factors
            const MlpFeatures &F = ip.feat;
            float v4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (F.var[i] >= 0) v4[i] = rv.vars[F.var[i]];
            const float clk = F.clock_var >= 0 ? rv.vars[F.clock_var] : 0.0f;
            float x[CSMC_MLP_IN];
            mlp_features(0, F, v4, clk, time, p.horizon, x);
            bool same = true;
#pragma unroll
            for (int i = 4; i < CSMC_MLP_IN; ++i) same = same && (__float_as_uint(x[i]) == x_last[i - 4]);
            if (!same) {  // warp-uniform: every lane holds the same features
                float theta[CSMC_MLP_CLASSES];
                if (TC) theta_tc(mlp, x, theta);
                else theta_exact(mlp, h1s, x, theta);
#pragma unroll
                for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) mfac[l] = tilt_factor(theta[l]);
#pragma unroll
                for (int i = 4; i < CSMC_MLP_IN; ++i) x_last[i - 4] = __float_as_uint(x[i]);
            }

            // the race: per-lane minima and sums, then the warp's
            LaneRace R;
            lane_race<TRACE, LOC8>(n, C, bits, rv, p.seed, run, step, mfac, R);
            unsigned long long best = R.best;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const unsigned long long o = __shfl_xor_sync(kFullWarp, best, off);
                best = o < best ? o : best;
            }
            const uint32_t win = bitrev_bits(static_cast<uint32_t>(best & 0xffffffffull), bits);
            const int owner = static_cast<int>(warp_lane_of(win));
            const float dmin = __shfl_sync(kFullWarp, R.bestd, owner);
            const float inv_w = __shfl_sync(kFullWarp, R.best_inv, owner);
            const float invp_w = __shfl_sync(kFullWarp, R.best_invp, owner);
            const bool tilted_w = __shfl_sync(kFullWarp, static_cast<int>(R.best_tilted), owner) != 0;
            const double rate_sum = warp_sum_d(R.rate_sum);
            const bool finite = static_cast<double>(dmin) < kDblMax;
            if (finite) {
                // step_log_ratio, with ln2 * log2(inv'_w / inv_w) of the last
                // tilted winner's (1/rate, 1/rate') pair reused
                const double ln2 = 0.6931471805599453;
                double r = d_mul(d_mul(ln2, rate_sum), static_cast<double>(dmin));
                if (tilted_w) {
                    if (__float_as_uint(inv_w) != w_inv || __float_as_uint(invp_w) != w_invp) {
                        w_inv = __float_as_uint(inv_w);
                        w_invp = __float_as_uint(invp_w);
                        w_term = d_mul(ln2, log2_d(d_div(static_cast<double>(invp_w), static_cast<double>(inv_w))));
                    }
                    r = d_add(r, w_term);
                }
                logw = d_add(logw, r);
            }
            if (TRACE) {
                double inv_sum[CSMC_MLP_CLASSES];
#pragma unroll
                for (int l = 0; l < CSMC_MLP_CLASSES; ++l) inv_sum[l] = warp_sum_d(R.inv_sum[l]);
                const uint32_t present = __reduce_or_sync(kFullWarp, R.cls_present);
                if (lane < CSMC_MLP_CLASSES) {  // lane l writes class l's row
                    const uint32_t wl = (rv.loc(n, win) - n.comp[win].loc_begin) & 3u;
                    const bool has = finite && ((present >> lane) & 1u);
                    const double s =
                        lane == 0 ? inv_sum[0] : (lane == 1 ? inv_sum[1] : (lane == 2 ? inv_sum[2] : inv_sum[3]));
                    MlpRow row;
#pragma unroll
                    for (int i = 0; i < CSMC_MLP_IN; ++i) row.x[i] = f_to_bf16(feat_of(x, lane, i));
                    row.a = has ? row_a(s, dmin, row_w) : 0.0f;
                    row.b = (has && tilted_w && wl == lane) ? row_w : 0.0f;
                    const uint64_t r = row0 + 4ull * step + lane;
                    if (r < ip.rows_cap) ip.rows[r] = row;
                    else atomicAdd(p.scratch + 4, 1ull);
                }
            }

            // the winner's transition (lane 0), then the time update
            int took = 0;
            if (lane == 0) {
                uint32_t s0 = step;
                float t0 = time;
                took = run_commit<false, SLOTS>(n, p.net.n_clocks, rv, sc, p.seed, p.var_id, run, s0, t0, win,
                                                      dmin);
            }
            __syncwarp();
            stale = __shfl_sync(kFullWarp, took, 0) != 0 || (p.net.n_clocks > 0 && finite);
            time = d2f(d_add(static_cast<double>(time), static_cast<double>(dmin)));
            ++step;
        }
    }
    if (lane == 0) {
        if (acc_hits) atomicAdd(p.scratch + 1, acc_hits);
        if (acc_steps) atomicAdd(p.scratch + 2, acc_steps);
        if (acc_capped) atomicAdd(p.scratch + 3, acc_capped);
    }
}

}  // namespace detail

template <bool TC, bool TRACE, bool SLOTS, bool LOC8>
int is_launch_one(const IsParams &p, int grid, int block, size_t smem, void *stream) {
    auto fn = detail::is_warp_kernel<TC, TRACE, SLOTS, LOC8>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool TC, bool TRACE, bool SLOTS, bool LOC8>
int is_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::is_warp_kernel<TC, TRACE, SLOTS, LOC8>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
