// Importance-sampling simulation: the thread-per-run kernel with every
// exponential delay drawn under the proposal network's tilt (csmc_mlp.h),
// the path's log-likelihood ratio carried in FP64, and a replay mode that
// writes the CE training rows of listed runs.
//
// Per step and run the proposal needs theta for each location class (local
// location index modulo 4).  Two kernels evaluate it:
//   * is_kernel (exact): four rows per lane on CUDA cores from FP32 copies of
//     the BF16 weights, in the operation order of mlp_theta, so runs are
//     bit-identical to the CPU oracle's;
//   * is_kernel_tc (tensor cores): the 32 lanes of a warp stage their 128
//     feature rows in shared memory and evaluate both hidden layers with
//     warp-level BF16 MMAs (mma.sync m16n8k16, FP32 accumulation): 64 + 256
//     MMAs per warp and step instead of ~20,000 FMAs per lane; the first
//     layer's accumulators become the second layer's operands in registers.
//     The lanes stay converged (runs end and restart between steps), and
//     theta differs from the exact evaluation only by accumulation order.
// Weights and estimates are exact for whichever theta a run used: the
// log-likelihood ratio is computed from the rates the run was drawn with.
// Replay mode writes exactly four rows per step of each listed run at a
// caller-given offset (rows of classes without a tilted component, and of
// steps in which nothing can fire, are zero-weighted), so the row set does
// not depend on scheduling.  Replay uses the kernel the runs were drawn
// with, so it follows the same paths.
#pragma once
#include "../include/csmc_mlp.h"
#include "sim_run.cuh"

namespace csmc {
namespace detail {

struct MlpSmem {  // the proposal network in shared memory
    float w1[CSMC_MLP_HID][CSMC_MLP_IN];        // FP32 copies (exact kernel)
    float w2[CSMC_MLP_HID][CSMC_MLP_HID];
    float b1[CSMC_MLP_HID], b2[CSMC_MLP_HID], w3[CSMC_MLP_HID];
    float b3, pad[3];
    uint16_t w1h[CSMC_MLP_HID][CSMC_MLP_IN];    // BF16 (tensor-core kernel)
    uint16_t w2h[CSMC_MLP_HID][CSMC_MLP_HID];
};

static __device__ __forceinline__ void stage_mlp(MlpSmem *m, const MlpParams *P) {
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID * CSMC_MLP_IN; i += blockDim.x) {
        (&m->w1h[0][0])[i] = (&P->w1[0][0])[i];
        (&m->w1[0][0])[i] = bf16_to_f((&P->w1[0][0])[i]);
    }
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID * CSMC_MLP_HID; i += blockDim.x) {
        (&m->w2h[0][0])[i] = (&P->w2[0][0])[i];
        (&m->w2[0][0])[i] = bf16_to_f((&P->w2[0][0])[i]);
    }
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID; i += blockDim.x) {
        m->b1[i] = P->b1[i];
        m->b2[i] = P->b2[i];
        m->w3[i] = P->w3[i];
    }
    if (threadIdx.x == 0) m->b3 = P->b3;
}

static __device__ __forceinline__ float clip_theta(float th) {
    return th < -CSMC_MLP_THETA_MAX ? -CSMC_MLP_THETA_MAX : (th > CSMC_MLP_THETA_MAX ? CSMC_MLP_THETA_MAX : th);
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
    return clip_theta(th);
}

// ---- tensor-core inference -------------------------------------------------

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

// theta for the four location classes of every lane of the warp.  Lane L's
// rows are 4L .. 4L+3 (class c = row mod 4), in m16 tile L/4; xs is the
// warp's staging area (128 rows x 16 BF16).  shared_x: this lane's features
// 4..15 (the class one-hot fills 0..3); inactive lanes stage zero rows.
static __device__ __noinline__ void warp_theta(const MlpSmem *m, uint32_t *xs, const float *shared_x, bool active,
                                               float *theta) {
    const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, tig = lane & 3u;
    __syncwarp();
#pragma unroll
    for (uint32_t c = 0; c < 4; ++c) {
#pragma unroll
        for (uint32_t w = 0; w < 8; ++w) {
            const uint32_t k0 = 2 * w, k1 = k0 + 1;
            const float v0 = !active ? 0.0f : (k0 < 4 ? (k0 == c ? 1.0f : 0.0f) : shared_x[k0]);
            const float v1 = !active ? 0.0f : (k1 < 4 ? (k1 == c ? 1.0f : 0.0f) : shared_x[k1]);
            xs[(4 * lane + c) * 8 + w] = pack_bf16(v0, v1);
        }
    }
    __syncwarp();
    for (uint32_t t = 0; t < 8; ++t) {
        const uint32_t r0 = 16 * t + g, r1 = r0 + 8;
        const uint32_t a0 = xs[r0 * 8 + tig], a1 = xs[r1 * 8 + tig], a2 = xs[r0 * 8 + tig + 4],
                       a3 = xs[r1 * 8 + tig + 4];
        uint32_t hA[4][4];  // second layer's A fragments, one per K step of 16
#pragma unroll
        for (uint32_t nt = 0; nt < 8; ++nt) {
            const uint16_t *wr = &m->w1h[8 * nt + g][0];
            float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            mma_16816(d, a0, a1, a2, a3, *reinterpret_cast<const uint32_t *>(wr + 2 * tig),
                      *reinterpret_cast<const uint32_t *>(wr + 2 * tig + 8));
            const uint32_t col = 8 * nt + 2 * tig;
            const float h00 = gelu_tc(d[0] + m->b1[col]), h01 = gelu_tc(d[1] + m->b1[col + 1]);
            const float h10 = gelu_tc(d[2] + m->b1[col]), h11 = gelu_tc(d[3] + m->b1[col + 1]);
            hA[nt >> 1][(nt & 1) * 2 + 0] = pack_bf16(h00, h01);
            hA[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16(h10, h11);
        }
        float s_lo = 0.0f, s_hi = 0.0f;
#pragma unroll
        for (uint32_t nt = 0; nt < 8; ++nt) {
            float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) {
                const uint16_t *wr = &m->w2h[8 * nt + g][16 * q];
                mma_16816(d, hA[q][0], hA[q][1], hA[q][2], hA[q][3], *reinterpret_cast<const uint32_t *>(wr + 2 * tig),
                          *reinterpret_cast<const uint32_t *>(wr + 2 * tig + 8));
            }
            const uint32_t col = 8 * nt + 2 * tig;
            s_lo = fmaf(gelu_tc(d[0] + m->b2[col]), m->w3[col], s_lo);
            s_lo = fmaf(gelu_tc(d[1] + m->b2[col + 1]), m->w3[col + 1], s_lo);
            s_hi = fmaf(gelu_tc(d[2] + m->b2[col]), m->w3[col], s_hi);
            s_hi = fmaf(gelu_tc(d[3] + m->b2[col + 1]), m->w3[col + 1], s_hi);
        }
        s_lo += __shfl_xor_sync(0xffffffffu, s_lo, 1);
        s_lo += __shfl_xor_sync(0xffffffffu, s_lo, 2);
        s_hi += __shfl_xor_sync(0xffffffffu, s_hi, 1);
        s_hi += __shfl_xor_sync(0xffffffffu, s_hi, 2);
        const float th_lo = clip_theta(m->b3 + s_lo), th_hi = clip_theta(m->b3 + s_hi);  // rows 16t+g, 16t+g+8
        const int j = static_cast<int>(lane) - 4 * static_cast<int>(t);
#pragma unroll
        for (uint32_t c = 0; c < 4; ++c) {
            const uint32_t r = 4u * (static_cast<uint32_t>(j) & 3u) + c;
            const uint32_t src = 4u * (r & 7u);
            const float vlo = __shfl_sync(0xffffffffu, th_lo, src), vhi = __shfl_sync(0xffffffffu, th_hi, src);
            if (j >= 0 && j < 4) theta[c] = r < 8 ? vlo : vhi;
        }
    }
    __syncwarp();
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

struct IsRace {
    unsigned long long best;
    float bestd, best_inv, best_invp;
    bool best_tilted;
    double rate_sum;                      // sum over tilted components of 1/inv' - 1/inv
    double inv_sum[CSMC_MLP_CLASSES];     // replay: per class, sum of 1/inv of tilted components
    uint32_t cls_present;                 // replay: bit l: class l has a tilted component
};

template <bool TRACE, bool LOC8>
static __device__ __forceinline__ IsRace is_race(const Net &n, uint32_t C, uint32_t bits, const RunView<LOC8> &rv,
                                                 uint64_t seed, uint64_t run, uint32_t step, const float *mfac) {
    IsRace R;
    R.best = ~0ull;
    R.bestd = R.best_inv = R.best_invp = 0.0f;
    R.best_tilted = false;
    R.rate_sum = 0.0;
#pragma unroll
    for (int l = 0; l < CSMC_MLP_CLASSES; ++l) R.inv_sum[l] = 0.0;
    R.cls_present = 0;
    for (uint32_t c = 0; c < C; c += 4) {
        const u32x4 blk = delay_block(seed, run, step, c >> 2);
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
                    R.rate_sum = d_add(R.rate_sum, rate_change(inv, invp));
                    if (TRACE) {
                        const double r = d_div(1.0, static_cast<double>(inv));
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
    return R;
}

// Replay rows of one step: four rows, features of each class, a and b.
template <bool LOC8>
static __device__ __forceinline__ void is_rows(MlpRow *rows, uint32_t step, const IsRace &R, bool finite,
                                               uint32_t win_class, const float *v4, uint32_t n_int, uint32_t C,
                                               float time, float horizon, float row_w) {
    float feat[CSMC_MLP_IN];
#pragma unroll
    for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) {
        mlp_features(l, v4, n_int, C, time, horizon, feat);
        MlpRow r;
#pragma unroll
        for (int i = 0; i < CSMC_MLP_IN; ++i) r.x[i] = f_to_bf16(feat[i]);
        const bool has = finite && ((R.cls_present >> l) & 1u);
        const double s = l == 0 ? R.inv_sum[0] : (l == 1 ? R.inv_sum[1] : (l == 2 ? R.inv_sum[2] : R.inv_sum[3]));
        r.a = has ? row_a(s, R.bestd, row_w) : 0.0f;
        r.b = (has && R.best_tilted && win_class == l) ? row_w : 0.0f;
        rows[4 * step + l] = r;
    }
}

#ifndef CSMC_IS_MIN_CTAS_PER_SM
#define CSMC_IS_MIN_CTAS_PER_SM 2
#endif

struct IsLane {  // one lane's current run
    bool have = false;
    unsigned long long ridx = 0;
    uint64_t run = 0;
    float time = 0.0f;
    uint32_t step = 0;
    double logw = 0.0;
    MlpRow *rows = nullptr;
    float row_w = 0.0f;
};

// Starts listed or numbered run ridx on a lane.
template <bool TRACE, bool SLOTS, bool LOC8>
static __device__ __forceinline__ void is_start(const IsParams &ip, const Net &n, uint32_t C, uint32_t V,
                                                const RunView<LOC8> &rv, RunScalars &sc, IsLane &L,
                                                unsigned long long ridx) {
    const SimParams &p = ip.s;
    L.have = true;
    L.ridx = ridx;
    if (TRACE) {
        L.run = p.first_run + ip.trace_runs[ridx];
        L.row_w = ip.trace_w[ridx];
        L.rows = ip.rows + ip.row_offset[ridx];
    } else {
        L.run = p.first_run + ridx;
    }
    run_init<SLOTS, LOC8>(n, C, V, rv, sc, p.var_id);
    L.time = 0.0f;
    L.step = 0;
    L.logw = 0.0;
}

// End of a run: outputs and counters; returns true when the run ended.
template <bool TRACE, bool LOC8>
static __device__ __forceinline__ bool is_finish(const IsParams &ip, const RunScalars &sc, IsLane &L,
                                                 unsigned long long &acc_hits, unsigned long long &acc_steps,
                                                 unsigned long long &acc_capped) {
    const SimParams &p = ip.s;
    const RunEnd e = run_end(sc, L.time, p.horizon, L.step, p.max_steps, p.loc_mode, p.is_max, p.threshold);
    if (!e.done) return false;
    if (!TRACE) {
        if (p.flags) p.flags[L.ridx] = static_cast<uint8_t>(e.flag);
        if (p.values) p.values[L.ridx] = e.value;
        if (p.steps) p.steps[L.ridx] = L.step;
        if (ip.logw) ip.logw[L.ridx] = L.logw;
        if (ip.wvals) ip.wvals[L.ridx] = e.flag ? exp2_d(d_mul(L.logw, 1.4426950408889634)) : 0.0;
    }
    acc_hits += e.flag;
    acc_steps += L.step;
    acc_capped += e.capped;
    L.have = false;
    return true;
}

// The race with the step's class factors, the likelihood ratio, replay rows,
// and the transition.
template <bool TRACE, bool SLOTS, bool LOC8>
static __device__ __forceinline__ void is_step(const IsParams &ip, const Net &n, uint32_t C, uint32_t bits,
                                               const RunView<LOC8> &rv, RunScalars &sc, IsLane &L, const float *mfac,
                                               const float *v4, uint32_t n_int) {
    const SimParams &p = ip.s;
    const IsRace R = is_race<TRACE, LOC8>(n, C, bits, rv, p.seed, L.run, L.step, mfac);
    const uint32_t win = bitrev_bits(static_cast<uint32_t>(R.best & 0xffffffffull), bits);
    const bool finite = static_cast<double>(R.bestd) < kDblMax;
    if (finite) L.logw = d_add(L.logw, step_log_ratio(R.rate_sum, R.bestd, R.best_tilted, R.best_inv, R.best_invp));
    if (TRACE) {
        const uint32_t wl = (rv.loc(n, win) - n.comp[win].loc_begin) & 3u;
        is_rows<LOC8>(L.rows, L.step, R, finite, wl, v4, n_int, C, L.time, p.horizon, L.row_w);
    }
    run_commit<false, SLOTS, LOC8>(n, p.net.n_clocks, rv, sc, p.seed, p.var_id, L.run, L.step, L.time, win, R.bestd);
}

// ---- exact kernel (CUDA-core inference, bit-identical to the oracle) --------
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
    IsLane L;
    RunScalars sc{0.0, 0.0, 0, 0, -1, 0, 0};

    for (;;) {
        const bool need = !L.have;
        const unsigned act = __activemask();
        const unsigned want = __ballot_sync(act, need);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if (static_cast<int>(lane) == leader)
                base = atomicAdd(p.scratch, static_cast<unsigned long long>(__popc(want)));
            base = __shfl_sync(act, base, leader);
            if (need) {
                const unsigned long long ridx = base + __popc(want & ((1u << lane) - 1u));
                if (ridx >= p.n_runs) break;
                is_start<TRACE, SLOTS, LOC8>(ip, n, C, V, rv, sc, L, ridx);
            }
        }
        if (is_finish<TRACE, LOC8>(ip, sc, L, acc_hits, acc_steps, acc_capped)) continue;

        run_receivers<false, SLOTS, LOC8>(n, C, V, rv, sc, p.seed, p.var_id, L.run, L.step);
        if (rate_table)
            for (uint32_t j = 0; j < P; ++j) rv.rates[j] = inv_rate(eval(n, rv.vars, n.rate_prog[j]));

        float v4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (uint32_t i = 0; i < n_int; ++i) v4[i] = rv.vars[i];
        float mfac[CSMC_MLP_CLASSES];
        float feat[CSMC_MLP_IN];
#pragma unroll
        for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) {
            mlp_features(l, v4, n_int, C, L.time, p.horizon, feat);
            mfac[l] = tilt_factor(mlp_theta_smem(mlp, feat));
        }
        is_step<TRACE, SLOTS, LOC8>(ip, n, C, bits, rv, sc, L, mfac, v4, n_int);
    }
    if (acc_hits) atomicAdd(p.scratch + 1, acc_hits);
    if (acc_steps) atomicAdd(p.scratch + 2, acc_steps);
    if (acc_capped) atomicAdd(p.scratch + 3, acc_capped);
}

// ---- tensor-core kernel: warp-converged steps --------------------------------
template <bool TRACE, bool SLOTS, bool LOC8>
__global__ void __launch_bounds__(128, CSMC_IS_MIN_CTAS_PER_SM) is_kernel_tc(const IsParams ip) {
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
    uint32_t *xs = reinterpret_cast<uint32_t *>(smem + p.blob_bytes + sizeof(MlpSmem)) + (t >> 5) * (128 * 8);
    uint8_t *st = smem + p.blob_bytes + sizeof(MlpSmem) + is_stage_bytes(T);
    const RunView<LOC8> rv = carve_run_view<LOC8>(st, V, P, C, T, t);

    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;
    IsLane L;
    RunScalars sc{0.0, 0.0, 0, 0, -1, 0, 0};
    bool exhausted = false;

    for (;;) {
        // refill; every lane stays in the loop until the whole warp is done
        const bool need = !L.have && !exhausted;
        const unsigned want = __ballot_sync(0xffffffffu, need);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if (static_cast<int>(lane) == leader)
                base = atomicAdd(p.scratch, static_cast<unsigned long long>(__popc(want)));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const unsigned long long ridx = base + __popc(want & ((1u << lane) - 1u));
                if (ridx >= p.n_runs) exhausted = true;
                else is_start<TRACE, SLOTS, LOC8>(ip, n, C, V, rv, sc, L, ridx);
            }
        }
        if (__all_sync(0xffffffffu, exhausted && !L.have)) break;
        bool active = L.have;
        if (active && is_finish<TRACE, LOC8>(ip, sc, L, acc_hits, acc_steps, acc_capped)) active = false;

        float v4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        float shared_x[CSMC_MLP_IN];
        if (active) {
            run_receivers<false, SLOTS, LOC8>(n, C, V, rv, sc, p.seed, p.var_id, L.run, L.step);
            if (rate_table)
                for (uint32_t j = 0; j < P; ++j) rv.rates[j] = inv_rate(eval(n, rv.vars, n.rate_prog[j]));
            for (uint32_t i = 0; i < n_int; ++i) v4[i] = rv.vars[i];
        }
        mlp_features(0, v4, n_int, C, L.time, p.horizon, shared_x);
        float theta[CSMC_MLP_CLASSES] = {0.0f, 0.0f, 0.0f, 0.0f};
        warp_theta(mlp, xs, shared_x, active, theta);
        if (active) {
            float mfac[CSMC_MLP_CLASSES];
#pragma unroll
            for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) mfac[l] = tilt_factor(theta[l]);
            is_step<TRACE, SLOTS, LOC8>(ip, n, C, bits, rv, sc, L, mfac, v4, n_int);
        }
    }
    if (acc_hits) atomicAdd(p.scratch + 1, acc_hits);
    if (acc_steps) atomicAdd(p.scratch + 2, acc_steps);
    if (acc_capped) atomicAdd(p.scratch + 3, acc_capped);
}

}  // namespace detail

template <bool TC, bool TRACE, bool SLOTS, bool LOC8>
int is_launch_one(const IsParams &p, int grid, int block, size_t smem, void *stream) {
    auto fn = TC ? detail::is_kernel_tc<TRACE, SLOTS, LOC8> : detail::is_kernel<TRACE, SLOTS, LOC8>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool TC, bool TRACE, bool SLOTS, bool LOC8>
int is_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = TC ? detail::is_kernel_tc<TRACE, SLOTS, LOC8> : detail::is_kernel<TRACE, SLOTS, LOC8>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
