// Thread-per-run simulation kernel for networks with race classes: the
// race reads one packed word per four components.
//
// Every component's location is kept as one byte, local index (5 bits) |
// delay code (3 bits): 0..3 the location's race class, 7 a location whose
// delay goes through its descriptor (zero-delay types, invariant-bounded or
// unclassed exponential locations), 6 padding past the last component.  The
// bytes of components 4q..4q+3 form word q of the thread's state, so one
// shared load gives the codes of the four components that share Philox
// block q.  A class member contributes only its key, (24-bit draw) * 256 +
// (255 - bit-reversed index), to the class's two largest keys; each class
// keeps four independent pairs, one per word of the Philox block (chain k),
// so consecutive members of a class do not wait on each other's shared-
// memory update.  After the components, the pairs of a class are merged and
// the class takes part in the race with its largest key, exactly as in
// race_classes (sim_run.cuh); the same cases fall back to race_exact.
//
// The Philox blocks of a step are computed through philox_step /
// philox_block (csmc_numeric.h): the counter words the blocks share are
// folded once per step, and the round keys are kernel parameters.  The
// per-step rate table is evaluated again only after a step that moved a
// component, unless a rate program reads a clock.
//
// Results are those of serial_kernel: the same draws, the same race
// outcome, the same transitions.
//
// Reference: simulation/simulation.cu:674-901 (simulation_kernel).
#pragma once
#include "sim_run.cuh"

namespace csmc {
namespace detail {

constexpr uint32_t kCodeGeneral = 7u;  // delay through the location's descriptor
constexpr uint32_t kCodePad = 6u;      // no component
constexpr uint32_t kKeyWords = 2u * 4u * CSMC_RACE_CLASSES;  // (largest, second) per chain per class

// Run state of one thread in the class-coded layout: vars[V] | rates[P] |
// shadow[V] (floats) | class keys (uint2 pairs [class*4 + chain]) |
// location words [ceil(C/4)] | slots[C] (u32); element i of thread t at
// [i * T + t] (the key pairs as 8-byte elements).
struct CodedView {
    VarView vars, rates, shadow;
    uint2 *keys;      // this thread's pair 0; stride T
    uint32_t *lw;     // this thread's location word 0; stride T
    uint32_t *slotv;  // this thread's element 0; stride T
    uint32_t T;

    __device__ __forceinline__ uint32_t byte_of(uint32_t c) const {
        return reinterpret_cast<const uint8_t *>(lw + (c >> 2) * T)[c & 3u];
    }
    // global location index of component c
    __device__ __forceinline__ uint32_t loc(const Net &n, uint32_t c) const {
        return n.comp[c].loc_begin + (byte_of(c) & 31u);
    }
    __device__ __forceinline__ void set_local(const Net &n, uint32_t c, uint32_t local) const {
        const uint32_t g = CSMC_DESC_CLASS(static_cast<uint32_t>(n.loc_desc[n.comp[c].loc_begin + local] >> 32));
        const uint32_t code = g < CSMC_RACE_CLASSES ? g : kCodeGeneral;
        reinterpret_cast<uint8_t *>(lw + (c >> 2) * T)[c & 3u] = static_cast<uint8_t>(local | (code << 5));
    }
};

static __host__ __device__ __forceinline__ uint32_t coded_words(uint32_t C) { return (C + 3u) >> 2; }

static __device__ __forceinline__ CodedView carve_coded_view(uint8_t *st, uint32_t V, uint32_t P, uint32_t C,
                                                             uint32_t T, uint32_t t) {
    float *fb = reinterpret_cast<float *>(st);
    CodedView r;
    r.vars = VarView{fb + t, T};
    r.rates = VarView{fb + V * T + t, T};
    r.shadow = VarView{fb + (V + P) * T + t, T};
    const uint32_t kb = (4u * (2u * V + P) * T + 7u) & ~7u;
    r.keys = reinterpret_cast<uint2 *>(st + kb) + t;
    const uint32_t lb = kb + 4u * kKeyWords * T;
    r.lw = reinterpret_cast<uint32_t *>(st + lb) + t;
    r.slotv = reinterpret_cast<uint32_t *>(st + lb + 4u * coded_words(C) * T) + t;
    r.T = T;
    return r;
}

// Delay of a component through its location's descriptor (the general
// path of race_exact).
static __device__ __forceinline__ float desc_delay(const Net &n, const CodedView &rv, uint32_t li, uint32_t x) {
    const uint64_t dsc = n.loc_desc[li];
    const uint32_t lo = static_cast<uint32_t>(dsc), fl = static_cast<uint32_t>(dsc >> 32);
    if (fl & CSMC_DESC_ZERO) return 0.0f;
    if (fl & (CSMC_DESC_INV | CSMC_DESC_EVAL)) return slow_delay(n, rv.vars, rv.rates, li, x);
    const float inv = (fl & CSMC_DESC_PROG) ? rv.rates[lo] : __uint_as_float(lo);
    return exp_delay(x, inv);
}

// The largest and second largest of four pairs (a_k largest, b_k second
// largest of chain k; keys of different chains are distinct).
static __device__ __forceinline__ void merge_chains(const uint2 &p0, const uint2 &p1, const uint2 &p2, const uint2 &p3,
                                                    uint32_t &m1, uint32_t &m2) {
    const uint32_t hi01 = max(p0.x, p1.x), lo01 = min(p0.x, p1.x);
    const uint32_t hi23 = max(p2.x, p3.x), lo23 = min(p2.x, p3.x);
    m1 = max(hi01, hi23);
    const uint32_t second_of_firsts = max(max(lo01, lo23), min(hi01, hi23));
    m2 = max(second_of_firsts, max(max(p0.y, p1.y), max(p2.y, p3.y)));
}

// The race decided from the class keys (race_classes' decision over the
// same keys); false: the caller runs race_exact.
static __device__ __forceinline__ bool race_coded(const Net &n, uint32_t C, uint32_t bits, uint32_t NG,
                                                  const CodedView &rv, const PhiloxKeys &K, uint64_t run,
                                                  uint32_t step, unsigned long long &best, float &bestd) {
    const uint32_t T = rv.T;
    for (uint32_t w = 0; w < 4u * NG; ++w) rv.keys[w * T] = make_uint2(0u, 0u);
    best = ~0ull;
    bestd = 0.0f;
    const PhiloxStep ps = philox_step(K, step, run);
    const uint32_t Q = coded_words(C);
    for (uint32_t q = 0; q < Q; ++q) {
        const u32x4 blk = philox_block(K, ps, q);
        const uint32_t wd = rv.lw[q * T];
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t b = (wd >> (8u * k)) & 0xffu;
            const uint32_t code = b >> 5;
            const uint32_t cc = 4u * q + k;
            const uint32_t x = word_of(blk, k);
            if (code < CSMC_RACE_CLASSES) {
                const uint32_t key = (x | 0xffu) - bitrev_bits(cc, bits);
                uint2 *pp = rv.keys + (code * 4u + k) * T;
                const uint2 m = *pp;
                *pp = make_uint2(max(m.x, key), max(m.y, min(m.x, key)));
            } else if (code == kCodeGeneral) {
                const float d = desc_delay(n, rv, n.comp[cc].loc_begin + (b & 31u), x);
                const unsigned long long key =
                    (static_cast<unsigned long long>(delay_key(d)) << 32) | bitrev_bits(cc, bits);
                if (key < best) {
                    best = key;
                    bestd = d;
                }
            }
        }
    }
    uint32_t inf_classes = 0;
    for (uint32_t g = 0; g < NG; ++g) {
        uint32_t a, second;
        merge_chains(rv.keys[(4u * g) * T], rv.keys[(4u * g + 1u) * T], rv.keys[(4u * g + 2u) * T],
                     rv.keys[(4u * g + 3u) * T], a, second);
        // key 0 (draw 0 at bit-reversed index 255) is also the "no member"
        // value; only component 255 of a 256-component network can hold it
        if (a == 0u && !(C == 256u && (rv.byte_of(255u) >> 5) == g)) continue;
        const uint32_t m1 = a >> 8, br1 = 255u - (a & 255u);
        const uint32_t li = rv.loc(n, bitrev_bits(br1, bits));
        const uint64_t dsc = n.loc_desc[li];
        const uint32_t lo = static_cast<uint32_t>(dsc), fl = static_cast<uint32_t>(dsc >> 32);
        const float inv = (fl & CSMC_DESC_PROG) ? rv.rates[lo] : __uint_as_float(lo);
        if (!(inv > 0.0f)) return false;  // delays 0, negative or NaN for the whole class
        if (!(inv <= 3.40282347e38f)) {   // +inf: the class's delays are +inf (NaN at u = 1)
            inf_classes |= 1u << g;
            continue;
        }
        const float d1 = exp_delay(m1 << 8, inv);
        if (m1 > 0 && second != 0u && exp_delay((m1 - 1u) << 8, inv) == d1) {
            const uint32_t m2 = second >> 8;
            if (m2 == m1 || exp_delay(m2 << 8, inv) == d1) return false;
        }
        const unsigned long long key = (static_cast<unsigned long long>(delay_key(d1)) << 32) | br1;
        if (key < best) {
            best = key;
            bestd = d1;
        }
    }
    if (inf_classes && static_cast<uint32_t>(best >> 32) >= delay_key(__uint_as_float(0x7f800000u))) return false;
    return true;
}

#ifndef CSMC_CODED_MIN_CTAS_PER_SM
#define CSMC_CODED_MIN_CTAS_PER_SM 4
#endif

template <bool VERIFY, bool SLOTS>
__global__ void __launch_bounds__(128, CSMC_CODED_MIN_CTAS_PER_SM) coded_kernel(const __grid_constant__ SimParams p) {
    extern __shared__ __align__(16) uint8_t smem[];
    stage_network(smem, p.blob, p.blob_bytes);
    const uint32_t C = p.net.n_comps, V = p.net.n_vars, P = p.net.n_rate_prog;
    const uint32_t T = blockDim.x, t = threadIdx.x;
    const CodedView rv = carve_coded_view(smem + p.blob_bytes, V, P, C, T, t);
    // padding bytes of the last location word never change
    if (C & 3u) rv.lw[(C >> 2) * T] = kCodePad * 0x20202020u;  // 0xc0 in every byte
    __syncthreads();
    const Net n = net_view(smem, p.net);
    const bool rate_table = (p.net.flags & CSMC_NET_RATE_TABLE) && P > 0;
    const bool rate_every_step = !(p.net.flags & CSMC_NET_RATE_NO_CLOCK);
    const uint32_t bits = ceil_log2(C);
    const uint32_t NG = p.net.n_classes;  // classes in use: only these keys are kept

    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;

    bool have = false;
    unsigned long long ridx = 0;
    uint64_t run = 0;
    float time = 0.0f;
    uint32_t step = 0;
    bool dirty = true;  // variables changed since the rate table was evaluated
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
                dirty = true;
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

        // ---- one step: receivers, rate table, race, commit
        if (run_receivers<VERIFY, SLOTS>(n, C, V, rv, sc, p.seed, p.var_id, run, step)) dirty = true;
        if (rate_table && (dirty || rate_every_step)) {
            for (uint32_t j = 0; j < P; ++j) rv.rates[j] = inv_rate(eval(n, rv.vars, n.rate_prog[j]));
            dirty = false;
        }
        unsigned long long best;
        float bestd;
        if (!race_coded(n, C, bits, NG, rv, p.keys, run, step, best, bestd))
            race_exact(n, C, bits, rv, p.seed, run, step, best, bestd);
        const uint32_t win = bitrev_bits(static_cast<uint32_t>(best & 0xffffffffull), bits);
        if (run_commit<VERIFY, SLOTS>(n, p.net.n_clocks, rv, sc, p.seed, p.var_id, run, step, time, win, bestd))
            dirty = true;
    }
    if (acc_hits) atomicAdd(p.scratch + 1, acc_hits);
    if (acc_steps) atomicAdd(p.scratch + 2, acc_steps);
    if (acc_capped) atomicAdd(p.scratch + 3, acc_capped);
}

}  // namespace detail

template <bool VERIFY, bool SLOTS>
int coded_launch_one(const SimParams &p, int grid, int block, size_t smem, void *stream) {
    auto fn = detail::coded_kernel<VERIFY, SLOTS>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool VERIFY, bool SLOTS>
int coded_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::coded_kernel<VERIFY, SLOTS>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
