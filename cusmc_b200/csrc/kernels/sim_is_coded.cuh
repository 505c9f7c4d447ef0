// Importance sampling, one thread per run, for networks whose exponential
// locations form race classes: the runs, draws, paths and FP64 log-
// likelihood ratios of is_warp_kernel (sim_is.cuh) with the CUDA-core
// evaluation of theta, at thread-per-run cost.
//
// Tilt groups.  Under the proposal a component's 1/rate is multiplied by
// its location class's factor (local index modulo 4), so the members of a
// race class in one location class share the tilted 1/rate: a (race class,
// location class) pair is a tilt group, and within a group the delay is a
// non-increasing function of the draw, as in the class-coded race of
// sim_coded.cuh.  The location byte's 3-bit code is the component's group
// (0..5), 7 for the descriptor path (locations of no race class, and pairs
// beyond the first six), 6 for padding.  The race keeps the largest key per
// group and chain, decides from the groups' largest draws and falls back to
// the full per-component race under the tilt where a flat spot of the delay
// could hide a tie.
//
// Log-likelihood ratio.  The step's sum of rate changes (1/inv' - 1/inv
// over tilted components) must carry the bits of the one-warp-per-run
// kernel, whose lane L sums the components of Philox blocks L, L + 32, ...
// in component order and whose lanes meet in a butterfly (csmc_mlp.h:
// warp_lane_of, warp_tree_d).  The butterfly over offsets 16, 8, 4, 2, 1 is
// the balanced binary tree over the lanes taken in 5-bit bit-reversed order,
// so the thread walks the lanes in that order (the race does not depend on
// the order of the blocks), sums each lane's blocks into its partial, and
// merges the partials with a five-level stack (a binary counter): the same
// additions in the same order.  A group member adds its group's rate
// change, computed once per step from the group's 1/rate and factor.
//
// Theta.  theta depends only on the run's features (the class one-hot
// aside) and the parameter block; a thread keeps its last features and
// class factors and needs new ones only when the features change.  It looks
// them up in a device-wide cache first; the misses are evaluated by the
// warp: the 32 lanes compute one feature row set together (theta_exact, the
// order of the oracle's mlp_theta), once per distinct pending feature
// vector of the warp, and the result goes into the cache.  Every lane of a
// warp stays in the loop until the whole warp has run out of runs.
#pragma once
#include <cstddef>

#include "sim_coded.cuh"
#include "sim_is.cuh"

// Up to 384 threads per CTA, at most 168 registers a thread (384 x 168
// fills the register file).  A 384-thread CTA keeps one copy of the
// network and the proposal for twelve warps (one CTA per SM); 128-thread
// CTAs fit two per SM (eight warps) within shared memory.
#ifndef CSMC_IS_CODED_MAX_THREADS
#define CSMC_IS_CODED_MAX_THREADS 384
#endif
#ifndef CSMC_IS_CODED_MIN_CTAS_PER_SM
#define CSMC_IS_CODED_MIN_CTAS_PER_SM 1
#endif

namespace csmc {
namespace detail {

// The CUDA-core evaluation reads only the FP32 copies at the start of
// MlpSmem: this kernel stages that prefix alone.
constexpr size_t kMlpExactBytes = offsetof(MlpSmem, w1h);
static_assert(kMlpExactBytes % 16 == 0, "the staging that follows stays 16-byte aligned");

static __device__ __forceinline__ void stage_mlp_exact(MlpSmem *m, const MlpParams *P) {
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID * CSMC_MLP_IN; i += blockDim.x)
        m->w1t[i % CSMC_MLP_IN][i / CSMC_MLP_IN] = bf16_to_f((&P->w1[0][0])[i]);
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID * CSMC_MLP_HID; i += blockDim.x)
        m->w2t[i % CSMC_MLP_HID][i / CSMC_MLP_HID] = bf16_to_f((&P->w2[0][0])[i]);
    for (uint32_t i = threadIdx.x; i < CSMC_MLP_HID; i += blockDim.x) {
        m->b1[i] = P->b1[i];
        m->b2[i] = P->b2[i];
        m->w3[i] = P->w3[i];
    }
    if (threadIdx.x == 0) m->b3 = P->b3;
}

// ---- the device-wide theta cache -------------------------------------------
// theta is a function of the feature vector and the parameter block alone,
// so class factors computed by one warp serve every later run with the same
// features.  An entry is written once per parameter generation: claimed by
// CAS on its state word (generation | busy bit), filled, then published by
// a release store of the generation; readers check the state with an
// acquire load, then compare the key.  Entries of other generations are
// free.  A lookup probes four consecutive entries.
constexpr uint32_t kThetaBusy = 0x80000000u;
constexpr uint32_t kThetaProbes = 4;

static __device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

static __device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

static __device__ __forceinline__ uint32_t theta_hash(uint32_t k0, uint32_t k1, uint32_t k2) {
    uint32_t h = (k0 * 0x9e3779b1u) ^ (k1 * 0x85ebca77u) ^ (k2 * 0xc2b2ae3du);
    h ^= h >> 15;
    h *= 0x2c1b3c6du;
    h ^= h >> 12;
    return h;
}

// true: mfac holds the cached factors of the features.  *slot: an entry the
// caller may claim for them after computing the factors (~0u: none).
static __device__ __noinline__ bool theta_lookup(const IsParams &ip, uint32_t k0, uint32_t k1, uint32_t k2,
                                                 float (&mfac)[CSMC_MLP_CLASSES], uint32_t &slot) {
    slot = ~0u;
    const uint32_t gen = ip.cache_gen;
    uint32_t i = theta_hash(k0, k1, k2) & ip.cache_mask;
    for (uint32_t probe = 0; probe < kThetaProbes; ++probe, i = (i + 1u) & ip.cache_mask) {
        uint32_t *e = ip.theta_cache + static_cast<size_t>(i) * CSMC_THETA_CACHE_WORDS;
        const uint32_t st = ld_acquire_u32(e);
        if (st == gen) {
            const uint4 a = *reinterpret_cast<const uint4 *>(e);
            if (a.y == k0 && a.z == k1 && a.w == k2) {
                const uint4 m = *reinterpret_cast<const uint4 *>(e + 4);
                mfac[0] = __uint_as_float(m.x);
                mfac[1] = __uint_as_float(m.y);
                mfac[2] = __uint_as_float(m.z);
                mfac[3] = __uint_as_float(m.w);
                return true;
            }
            continue;
        }
        if (st == (gen | kThetaBusy)) continue;  // being written (its key unknown yet)
        slot = i;                                // free for this generation
        return false;
    }
    return false;
}

static __device__ __noinline__ void theta_insert(const IsParams &ip, uint32_t slot, uint32_t k0, uint32_t k1,
                                                 uint32_t k2, const float (&mfac)[CSMC_MLP_CLASSES]) {
    const uint32_t gen = ip.cache_gen;
    uint32_t *e = ip.theta_cache + static_cast<size_t>(slot) * CSMC_THETA_CACHE_WORDS;
    const uint32_t old = ld_acquire_u32(e);
    if (old == gen || old == (gen | kThetaBusy)) return;  // taken meanwhile
    if (atomicCAS(e, old, gen | kThetaBusy) != old) return;
    e[1] = k0;
    e[2] = k1;
    e[3] = k2;
    *reinterpret_cast<uint4 *>(e + 4) =
        make_uint4(__float_as_uint(mfac[0]), __float_as_uint(mfac[1]), __float_as_uint(mfac[2]),
                   __float_as_uint(mfac[3]));
    st_release_u32(e, gen);
}

// theta of NV feature vectors at once (keys: BF16 bits of features 4..9
// packed in pairs): the operations of theta_exact (sim_is.cuh) for each of
// the 4 NV rows in the same order, with every weight read once for all
// rows.  h1s: the warp's staging, 1 KB per vector.
template <int NV>
static __device__ __forceinline__ void theta_exact_n(const MlpSmem *m, float *h1s, const uint32_t (&key)[NV][3],
                                                     float (&theta)[NV][CSMC_MLP_CLASSES]) {
    const uint32_t lane = threadIdx.x & 31u;
    float x[NV][CSMC_MLP_IN];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int i = 0; i < CSMC_MLP_IN; ++i) x[v][i] = 0.0f;
#pragma unroll
        for (int w = 0; w < 3; ++w) {
            x[v][4 + 2 * w] = __uint_as_float(key[v][w] << 16);
            x[v][5 + 2 * w] = __uint_as_float(key[v][w] & 0xffff0000u);
        }
    }
    float za[NV][4], zb[NV][4];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            za[v][r] = m->b1[lane];
            zb[v][r] = m->b1[lane + 32];
        }
#pragma unroll
    for (int i = 0; i < CSMC_MLP_IN; ++i) {
        const float wa = m->w1t[i][lane], wb = m->w1t[i][lane + 32];
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
            for (uint32_t r = 0; r < 4; ++r) {
                const float xi = feat_of(x[v], r, i);
                za[v][r] = f_fma(xi, wa, za[v][r]);
                zb[v][r] = f_fma(xi, wb, zb[v][r]);
            }
    }
    __syncwarp();  // the previous evaluation's readers of h1s are done
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        float4 *h4 = reinterpret_cast<float4 *>(h1s + v * (CSMC_MLP_HID * 4));
        h4[lane] = make_float4(bf16_round(gelu_f(za[v][0])), bf16_round(gelu_f(za[v][1])),
                               bf16_round(gelu_f(za[v][2])), bf16_round(gelu_f(za[v][3])));
        h4[lane + 32] = make_float4(bf16_round(gelu_f(zb[v][0])), bf16_round(gelu_f(zb[v][1])),
                                    bf16_round(gelu_f(zb[v][2])), bf16_round(gelu_f(zb[v][3])));
    }
    __syncwarp();
    float ya[NV][4], yb[NV][4];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            ya[v][r] = m->b2[lane];
            yb[v][r] = m->b2[lane + 32];
        }
#pragma unroll 4
    for (int j = 0; j < CSMC_MLP_HID; ++j) {
        const float wa = m->w2t[j][lane], wb = m->w2t[j][lane + 32];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const float4 h = reinterpret_cast<const float4 *>(h1s + v * (CSMC_MLP_HID * 4))[j];
            ya[v][0] = f_fma(h.x, wa, ya[v][0]);
            ya[v][1] = f_fma(h.y, wa, ya[v][1]);
            ya[v][2] = f_fma(h.z, wa, ya[v][2]);
            ya[v][3] = f_fma(h.w, wa, ya[v][3]);
            yb[v][0] = f_fma(h.x, wb, yb[v][0]);
            yb[v][1] = f_fma(h.y, wb, yb[v][1]);
            yb[v][2] = f_fma(h.z, wb, yb[v][2]);
            yb[v][3] = f_fma(h.w, wb, yb[v][3]);
        }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            float s = f_fma(gelu_f(yb[v][r]), m->w3[lane + 32], f_fma(gelu_f(ya[v][r]), m->w3[lane], 0.0f));
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) s = f_add(s, __shfl_xor_sync(kFullWarp, s, off));
            theta[v][r] = clip_theta(f_add(m->b3, s));
        }
}

// Distinct feature vectors per warp evaluation: evaluating two at once
// (every weight read once for eight rows) measured no faster than one.
constexpr int kThetaBatch = 1;

// The class-coded view with the tilt groups' location codes.
struct IsCodedView : CodedView {
    uint64_t map;  // IsParams::group_map
    __device__ __forceinline__ void set_local(const Net &n, uint32_t c, uint32_t local) const {
        const uint32_t g = CSMC_DESC_CLASS(static_cast<uint32_t>(n.loc_desc[n.comp[c].loc_begin + local] >> 32));
        const uint32_t code = g < CSMC_RACE_CLASSES ? static_cast<uint32_t>(map >> (3u * (4u * g + (local & 3u)))) & 7u
                                                    : kCodeGeneral;
        reinterpret_cast<uint8_t *>(lw + (c >> 2) * T)[c & 3u] = static_cast<uint8_t>(local | (code << 5));
    }
};

// Per thread and group: the step's 1/rate and 1/rate' bits and the rate
// change 1/inv' - 1/inv (FP64, as two words); element i at [i * T].
struct GroupRates {
    uint32_t *w;  // this thread's group 0 word 0; group gi word j at [(4 gi + j) * T]
    uint32_t T;
    __device__ __forceinline__ float inv(uint32_t gi) const { return __uint_as_float(w[(4u * gi) * T]); }
    __device__ __forceinline__ float invp(uint32_t gi) const { return __uint_as_float(w[(4u * gi + 1u) * T]); }
    __device__ __forceinline__ double diff(uint32_t gi) const {
        return __hiloint2double(static_cast<int>(w[(4u * gi + 3u) * T]), static_cast<int>(w[(4u * gi + 2u) * T]));
    }
    __device__ __forceinline__ void set(uint32_t gi, float inv, float invp, double diff) const {
        w[(4u * gi) * T] = __float_as_uint(inv);
        w[(4u * gi + 1u) * T] = __float_as_uint(invp);
        w[(4u * gi + 2u) * T] = static_cast<uint32_t>(__double2loint(diff));
        w[(4u * gi + 3u) * T] = static_cast<uint32_t>(__double2hiint(diff));
    }
};

// A component's delay through its location's descriptor under the tilt
// factor m (the general path of lane_race in sim_is.cuh).
static __device__ __forceinline__ float is_desc_delay(const Net &n, VarView vars, VarView rates, uint32_t li,
                                                      uint32_t x, float m, bool &tilted, float &inv, float &invp) {
    const uint64_t dsc = n.loc_desc[li];
    const uint32_t lo = static_cast<uint32_t>(dsc), fl = static_cast<uint32_t>(dsc >> 32);
    tilted = false;
    inv = invp = 0.0f;
    if (fl & CSMC_DESC_ZERO) return 0.0f;
    if (fl & (CSMC_DESC_INV | CSMC_DESC_EVAL)) return is_slow_delay(n, vars, rates, li, x, m, &tilted, &inv, &invp);
    inv = (fl & CSMC_DESC_PROG) ? rates[lo] : __uint_as_float(lo);
    invp = inv;
    if (tiltable(inv)) {
        invp = f_mul(inv, m);
        tilted = true;
    }
    return exp_delay(x, invp);
}

static __device__ __forceinline__ float mfac_of(const float (&mfac)[CSMC_MLP_CLASSES], uint32_t l) {
    return l == 0 ? mfac[0] : (l == 1 ? mfac[1] : (l == 2 ? mfac[2] : mfac[3]));
}

// The race's winner data.
struct IsBest {
    unsigned long long key;
    float d, inv, invp;
    bool tilted;
};

static __device__ __forceinline__ void is_take(IsBest &b, unsigned long long key, float d, float inv, float invp,
                                               bool tilted) {
    if (key < b.key) {
        b.key = key;
        b.d = d;
        b.inv = inv;
        b.invp = invp;
        b.tilted = tilted;
    }
}

// One component's part in the race and in its lane's partial sum.  cb:
// 255 minus the component's bit-reversed index, the low byte of its group
// key.  ALLG: every component is a group member (no descriptor path, no
// padding).
template <bool ALLG, uint32_t k>
static __device__ __forceinline__ void is_member(const Net &n, const IsCodedView &rv, const GroupRates &gr,
                                                 uint32_t NG, uint32_t tilt_mask, const float (&mfac)[CSMC_MLP_CLASSES],
                                                 uint32_t wd, uint32_t cc, uint32_t x, uint32_t cb, IsBest &best,
                                                 double &part) {
    const uint32_t b = (wd >> (8u * k)) & 0xffu;
    const uint32_t code = b >> 5;
    const uint32_t T = rv.T;
    if (ALLG || code < NG) {
        const uint32_t key = (x & 0xffffff00u) | cb;
        uint32_t *pp = rv.keys + (code * 4u + k) * T;
        *pp = max(*pp, key);
        if ((tilt_mask >> code) & 1u) part = d_add(part, gr.diff(code));
    } else if (code == kCodeGeneral) {
        const uint32_t local = b & 31u;
        bool tl;
        float inv, invp;
        const float d = is_desc_delay(n, rv.vars, rv.rates, n.comp[cc].loc_begin + local, x, mfac_of(mfac, local & 3u),
                                      tl, inv, invp);
        is_take(best, (static_cast<unsigned long long>(delay_key(d)) << 32) | (255u - cb), d, inv, invp, tl);
        if (tl) part = d_add(part, rate_change(inv, invp));
    }
}

// The full race under the tilt, one delay per component (the decision of
// lane_race); used where the groups' largest keys do not decide the step.
static __device__ __noinline__ void is_race_exact(const Net &n, uint32_t C, uint32_t bits, const IsCodedView &rv,
                                                  const GroupRates &gr, uint32_t NG,
                                                  const float (&mfac)[CSMC_MLP_CLASSES], uint64_t seed, uint64_t run,
                                                  uint32_t step, IsBest &best) {
    best.key = ~0ull;
    best.d = best.inv = best.invp = 0.0f;
    best.tilted = false;
    for (uint32_t c = 0; c < C; c += 4) {
        const u32x4 blk = delay_block(seed, run, step, c >> 2);
        const uint32_t wd = rv.lw[(c >> 2) * rv.T];
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t cc = c + k;
            if (cc >= C) break;
            const uint32_t b = (wd >> (8u * k)) & 0xffu;
            const uint32_t code = b >> 5, local = b & 31u;
            const uint32_t x = word_of(blk, k);
            float d, inv, invp;
            bool tl;
            if (code < NG) {
                inv = gr.inv(code);
                invp = gr.invp(code);
                tl = tiltable(inv);
                d = exp_delay(x, invp);
            } else {
                d = is_desc_delay(n, rv.vars, rv.rates, n.comp[cc].loc_begin + local, x, mfac_of(mfac, local & 3u), tl,
                                  inv, invp);
            }
            is_take(best, (static_cast<unsigned long long>(delay_key(d)) << 32) | bitrev_bits(cc, bits), d, inv, invp,
                    tl);
        }
    }
}

// One merge step of the butterfly stack: leaf i (0..31, lanes in 5-bit
// bit-reversed order) with value v; returns true with the total in v after
// the last leaf.
static __device__ __forceinline__ void tree_push(uint32_t i, double v, double (&s)[5], double &total) {
    if (!(i & 1u)) { s[0] = v; return; }
    v = d_add(s[0], v);
    if (!(i & 2u)) { s[1] = v; return; }
    v = d_add(s[1], v);
    if (!(i & 4u)) { s[2] = v; return; }
    v = d_add(s[2], v);
    if (!(i & 8u)) { s[3] = v; return; }
    v = d_add(s[3], v);
    if (!(i & 16u)) { s[4] = v; return; }
    total = d_add(s[4], v);
}

// The step's race and sum of rate changes.  Returns false when the groups'
// keys do not decide the race (the caller runs is_race_exact); `sum` is
// valid either way.
template <bool ALLG>
static __device__ __forceinline__ bool is_race_coded(const Net &n, uint32_t C, uint32_t bits, uint32_t NG,
                                                     uint32_t tilt_mask, const IsCodedView &rv, const GroupRates &gr,
                                                     const float (&mfac)[CSMC_MLP_CLASSES], const PhiloxKeys &K,
                                                     uint64_t run, uint32_t step, IsBest &best, double &sum) {
    const uint32_t T = rv.T;
    for (uint32_t w = 0; w < 4u * NG; ++w) rv.keys[w * T] = 0u;
    best.key = ~0ull;
    best.d = best.inv = best.invp = 0.0f;
    best.tilted = false;
    const PhiloxStep ps = philox_step(K, step, run);
    const uint32_t hi_shift = bits - 2u;  // bits >= 2: at least four components
    const uint32_t nb = (C + 3u) >> 2;
    double stack[5];
    sum = 0.0;
    for (uint32_t i = 0; i < CSMC_WARP; ++i) {
        const uint32_t L = __brev(i) >> 27;  // the lane whose partial is leaf i of the butterfly
        double part = 0.0;
        for (uint32_t q = L; q < nb; q += CSMC_WARP) {
            const u32x4 blk = philox_block(K, ps, q);
            const uint32_t wd = rv.lw[q * T], cc = 4u * q;
            const uint32_t rq = hi_shift ? (__brev(q) >> (32u - hi_shift)) : 0u;
            const uint32_t cb = 255u - rq;
            is_member<ALLG, 0>(n, rv, gr, NG, tilt_mask, mfac, wd, cc, blk.x, cb, best, part);
            is_member<ALLG, 1>(n, rv, gr, NG, tilt_mask, mfac, wd, cc + 1u, blk.y, cb - (2u << hi_shift), best, part);
            is_member<ALLG, 2>(n, rv, gr, NG, tilt_mask, mfac, wd, cc + 2u, blk.z, cb - (1u << hi_shift), best, part);
            is_member<ALLG, 3>(n, rv, gr, NG, tilt_mask, mfac, wd, cc + 3u, blk.w, cb - (3u << hi_shift), best, part);
        }
        tree_push(i, part, stack, sum);
    }
    // each group races with its largest key under its tilted 1/rate
    uint32_t inf_groups = 0, ties = 0;
    uint32_t top[CSMC_IS_GROUPS];
    float dg[CSMC_IS_GROUPS];
#pragma unroll
    for (uint32_t g = 0; g < CSMC_IS_GROUPS; ++g) {
        top[g] = 0u;
        dg[g] = 0.0f;
        if (g >= NG) continue;
        const uint32_t *kg = rv.keys + (4u * g) * T;
        const uint32_t a = max(max(kg[0], kg[T]), max(kg[2u * T], kg[3u * T]));
        // key 0 (draw 0 at bit-reversed index 255) is also the "no member"
        // value; only component 255 of a 256-component network can hold it
        if (a == 0u && !(C == 256u && (rv.byte_of(255u) >> 5) == g)) continue;
        const float invp = gr.invp(g);
        if (!(invp > 0.0f)) return false;  // delays 0, negative or NaN for the whole group
        if (!(invp <= 3.40282347e38f)) {    // +inf: the group's delays are +inf (NaN at u = 1)
            inf_groups |= 1u << g;
            continue;
        }
        const uint32_t m1 = a >> 8, br1 = 255u - (a & 255u);
        const float d1 = exp_delay(m1 << 8, invp);
        top[g] = a;
        dg[g] = d1;
        ties |= m1 > 0u ? (1u << g) : 0u;
        const float inv = gr.inv(g);
        is_take(best, (static_cast<unsigned long long>(delay_key(d1)) << 32) | br1, d1, inv, invp, tiltable(inv));
    }
    // a flat spot at a minimal group's largest draw could hide a member
    // with a smaller index and the same delay: the exact race decides
#pragma unroll
    for (uint32_t g = 0; g < CSMC_IS_GROUPS; ++g) {
        if (!((ties >> g) & 1u) || dg[g] != best.d) continue;
        if (exp_delay(((top[g] >> 8) - 1u) << 8, gr.invp(g)) == dg[g]) return false;
    }
    if (inf_groups && static_cast<uint32_t>(best.key >> 32) >= delay_key(__uint_as_float(0x7f800000u))) return false;
    return true;
}

template <bool SLOTS, bool ALLG>
__global__ void __launch_bounds__(CSMC_IS_CODED_MAX_THREADS, CSMC_IS_CODED_MIN_CTAS_PER_SM)
    is_coded_kernel(const __grid_constant__ IsParams ip) {
    const SimParams &p = ip.s;
    extern __shared__ __align__(16) uint8_t smem[];
    stage_network(smem, p.blob, p.blob_bytes);
    MlpSmem *mlp = reinterpret_cast<MlpSmem *>(smem + p.blob_bytes);
    stage_mlp_exact(mlp, ip.mlp);
    const uint32_t C = p.net.n_comps, V = p.net.n_vars, P = p.net.n_rate_prog;
    const uint32_t T = blockDim.x, t = threadIdx.x, lane = t & 31u;
    const uint32_t NG = ip.n_groups;
    uint8_t *h1_base = smem + p.blob_bytes + kMlpExactBytes;
    float *h1s = reinterpret_cast<float *>(h1_base) + (t >> 5) * (kThetaBatch * CSMC_MLP_HID * CSMC_MLP_CLASSES);
    uint8_t *slab = h1_base + (T >> 5) * (4u * kThetaBatch * CSMC_MLP_HID * CSMC_MLP_CLASSES);
    const GroupRates gr{reinterpret_cast<uint32_t *>(slab) + t, T};
    const bool recv = (p.net.recv_lo | p.net.recv_hi) != 0;
    IsCodedView rv;
    static_cast<CodedView &>(rv) = carve_coded_view(slab + 16u * NG * T, V, P, C, NG, recv, T, t);
    rv.map = ip.group_map;
    if (C & 3u) rv.lw[(C >> 2) * T] = kCodePad * 0x20202020u;  // padding bytes never change
    __syncthreads();
    const Net n = net_view(smem, p.net);
    const bool rate_table = (p.net.flags & CSMC_NET_RATE_TABLE) && P > 0;
    const uint32_t bits = ceil_log2(C);
    const MlpFeatures &F = ip.feat;

    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;
    bool have = false, exhausted = false;
    unsigned long long ridx = 0;
    uint64_t run = 0;
    float time = 0.0f;
    uint32_t step = 0;
    double logw = 0.0;
    bool stale = true;
    RunScalars sc{0.0, 0.0, 0, 0, -1, 0, 0};
    // the last evaluated features (BF16 bits of x[4..9], packed in pairs)
    // and their class factors, kept across steps and runs
    uint32_t lk0 = 0, lk1 = 0, lk2 = 0;
    bool theta_valid = false;
    float mfac[CSMC_MLP_CLASSES] = {1.0f, 1.0f, 1.0f, 1.0f};
    bool rates_changed = true;  // the groups' rates need a new look
    uint32_t gvalid = 0;        // groups whose GroupRates entry has been written
    // the last tilted winner's 1/rate and 1/rate' bits and its log term
    uint32_t w_inv = 0xffffffffu, w_invp = 0xffffffffu;
    double w_term = 0.0;

    for (;;) {
        // ---- refill lanes whose run ended from the work counter
        const bool need_run = !have && !exhausted;
        const unsigned want = __ballot_sync(kFullWarp, need_run);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if (static_cast<int>(lane) == leader)
                base = atomicAdd(p.scratch, static_cast<unsigned long long>(__popc(want)));
            base = __shfl_sync(kFullWarp, base, leader);
            if (need_run) {
                ridx = base + __popc(want & ((1u << lane) - 1u));
                if (ridx >= p.n_runs) {
                    exhausted = true;
                } else {
                    have = true;
                    run = p.first_run + ridx;
                    run_init<SLOTS>(n, C, V, rv, sc, p.var_id);
                    time = 0.0f;
                    step = 0;
                    logw = 0.0;
                    stale = true;
                }
            }
        }
        if (__all_sync(kFullWarp, exhausted)) break;

        // ---- end of run
        if (have) {
            const RunEnd e = run_end(sc, time, p.horizon, step, p.max_steps, p.loc_mode, p.is_max, p.threshold);
            if (e.done) {
                if (p.flags) p.flags[ridx] = static_cast<uint8_t>(e.flag);
                if (p.values) p.values[ridx] = e.value;
                if (p.steps) p.steps[ridx] = step;
                if (ip.logw) ip.logw[ridx] = logw;
                if (ip.wvals) ip.wvals[ridx] = e.flag ? exp2_d(d_mul(logw, 1.4426950408889634)) : 0.0;
                acc_hits += e.flag;
                acc_steps += step;
                acc_capped += e.capped;
                have = false;
            }
        }

        // ---- receivers and the rate table (this thread's run)
        uint32_t fk0 = 0, fk1 = 0, fk2 = 0;
        bool need_theta = false;
        if (have) {
            if (run_receivers<false, SLOTS>(n, C, V, rv, sc, p.seed, p.var_id, run, step)) stale = true;
            if (rate_table && stale) {
                for (uint32_t j = 0; j < P; ++j) rv.rates[j] = inv_rate(eval(n, rv.vars, n.rate_prog[j]));
                rates_changed = true;
            }
            stale = false;
            float v4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (F.var[i] >= 0) v4[i] = rv.vars[F.var[i]];
            const float clk = F.clock_var >= 0 ? rv.vars[F.clock_var] : 0.0f;
            float x[CSMC_MLP_IN];
            mlp_features(0, F, v4, clk, time, p.horizon, x);
            fk0 = (f_bits(x[4]) >> 16) | (f_bits(x[5]) & 0xffff0000u);
            fk1 = (f_bits(x[6]) >> 16) | (f_bits(x[7]) & 0xffff0000u);
            fk2 = (f_bits(x[8]) >> 16) | (f_bits(x[9]) & 0xffff0000u);
            need_theta = !theta_valid || fk0 != lk0 || fk1 != lk1 || fk2 != lk2;
        }

        // ---- theta for the lanes whose features changed: the cache, then
        // one distinct feature vector at a time evaluated by the whole warp
        uint32_t slot = ~0u;
        if (need_theta && ip.theta_cache) {
            float mc[CSMC_MLP_CLASSES];
            if (theta_lookup(ip, fk0, fk1, fk2, mc, slot)) {
#pragma unroll
                for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) mfac[l] = mc[l];
                lk0 = fk0;
                lk1 = fk1;
                lk2 = fk2;
                theta_valid = true;
                need_theta = false;
                rates_changed = true;
            }
        }
        unsigned pend = __ballot_sync(kFullWarp, need_theta);
        while (pend) {
            const int j = __ffs(pend) - 1;
            uint32_t key[1][3] = {{__shfl_sync(kFullWarp, fk0, j), __shfl_sync(kFullWarp, fk1, j),
                                   __shfl_sync(kFullWarp, fk2, j)}};
            float theta[1][CSMC_MLP_CLASSES];
            theta_exact_n<1>(mlp, h1s, key, theta);
            const bool mine = need_theta && fk0 == key[0][0] && fk1 == key[0][1] && fk2 == key[0][2];
            if (mine) {
#pragma unroll
                for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) mfac[l] = tilt_factor(theta[0][l]);
                lk0 = fk0;
                lk1 = fk1;
                lk2 = fk2;
                theta_valid = true;
                need_theta = false;
                rates_changed = true;
                if (static_cast<int>(lane) == j && slot != ~0u) theta_insert(ip, slot, fk0, fk1, fk2, mfac);
            }
            pend &= ~__ballot_sync(kFullWarp, mine);
        }
        if (!have) continue;

        // ---- the groups' tilted rates and rate changes
        uint32_t tilt_mask = 0;
        for (uint32_t g = 0; g < NG; ++g) {
            const uint32_t sg = ip.group_src[g];
            const float inv = (sg & CSMC_CLASS_SRC_PROG) ? rv.rates[sg & 0xffffu] : __uint_as_float(sg);
            const bool tl = tiltable(inv);
            tilt_mask |= tl ? (1u << g) : 0u;
            if (rates_changed) {
                const float invp = tl ? f_mul(inv, mfac_of(mfac, (ip.group_l >> (2u * g)) & 3u)) : inv;
                if (!((gvalid >> g) & 1u) || __float_as_uint(inv) != __float_as_uint(gr.inv(g)) ||
                    __float_as_uint(invp) != __float_as_uint(gr.invp(g))) {
                    gr.set(g, inv, invp, tl ? rate_change(inv, invp) : 0.0);
                    gvalid |= 1u << g;
                }
            }
        }
        rates_changed = false;

        // ---- the race, the log-likelihood ratio, the winner's transition
        IsBest best;
        double rsum;
        if (!is_race_coded<ALLG>(n, C, bits, NG, tilt_mask, rv, gr, mfac, p.keys, run, step, best, rsum))
            is_race_exact(n, C, bits, rv, gr, NG, mfac, p.seed, run, step, best);
        const uint32_t win = bitrev_bits(static_cast<uint32_t>(best.key & 0xffffffffull), bits);
        const float dmin = best.d;
        const bool finite = static_cast<double>(dmin) < kDblMax;
        if (finite) {
            const double ln2 = 0.6931471805599453;
            double r = d_mul(d_mul(ln2, rsum), static_cast<double>(dmin));
            if (best.tilted) {
                if (__float_as_uint(best.inv) != w_inv || __float_as_uint(best.invp) != w_invp) {
                    w_inv = __float_as_uint(best.inv);
                    w_invp = __float_as_uint(best.invp);
                    w_term =
                        d_mul(ln2, log2_d(d_div(static_cast<double>(best.invp), static_cast<double>(best.inv))));
                }
                r = d_add(r, w_term);
            }
            logw = d_add(logw, r);
        }
        const bool took = run_commit<false, SLOTS>(n, p.net.n_clocks, rv, sc, p.seed, p.var_id, run, step, time, win,
                                                   dmin);
        stale = took || (p.net.n_clocks > 0 && finite);
    }
    if (acc_hits) atomicAdd(p.scratch + 1, acc_hits);
    if (acc_steps) atomicAdd(p.scratch + 2, acc_steps);
    if (acc_capped) atomicAdd(p.scratch + 3, acc_capped);
}

}  // namespace detail

template <bool SLOTS, bool ALLG>
int is_coded_launch_one(const IsParams &p, int grid, int block, size_t smem, void *stream) {
    auto fn = detail::is_coded_kernel<SLOTS, ALLG>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool SLOTS, bool ALLG>
int is_coded_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::is_coded_kernel<SLOTS, ALLG>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
