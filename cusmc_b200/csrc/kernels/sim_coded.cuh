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
// (255 - bit-reversed index), to its class's largest key; each class keeps
// four independent maxima, one per word of the Philox block (chain k), so
// consecutive members of a class do not wait on each other's shared-memory
// update.  After the components, the chains of a class are merged and the
// class takes part in the race with its largest key, as in race_classes
// (sim_run.cuh).  Where race_classes consults the second largest key (a
// lower draw that rounds to the same float delay could hide a member with a
// smaller index), this kernel falls back to race_exact whenever the largest
// draw of a class whose delay is the race's minimum sits on such a flat
// spot of the delay function (about 2e-4 .. 4e-3 per step for a class of
// 1-10 members, far less with many); delays do not increase with the
// draw, so no flat spot means no tie with a lower draw.
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
#ifndef CSMC_CODED_UNROLL
#define CSMC_CODED_UNROLL 1
#endif
constexpr int kCodedUnroll = CSMC_CODED_UNROLL;  // Philox blocks of the race loop in flight per iteration

// Run state of one thread in the class-coded layout: vars[V] | rates[P] |
// shadow[V] (floats; only for networks with receiving edges, else the
// snapshot view aliases the variables and is never used) | class keys
// ([class*4 + chain], NG classes) | location words [ceil(C/4)] | slots[C]
// (all 4-byte words); element i of thread t at [i * T + t].
struct CodedView {
    VarView vars, rates, shadow;
    uint32_t *keys;   // this thread's chain 0 of class 0; stride T
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
                                                             uint32_t NG, bool recv, uint32_t T, uint32_t t) {
    float *fb = reinterpret_cast<float *>(st);
    CodedView r;
    r.vars = VarView{fb + t, T};
    r.rates = VarView{fb + V * T + t, T};
    r.shadow = recv ? VarView{fb + (V + P) * T + t, T} : r.vars;
    const uint32_t kb = 4u * ((recv ? 2u : 1u) * V + P) * T;
    r.keys = reinterpret_cast<uint32_t *>(st + kb) + t;
    const uint32_t lb = kb + 4u * 4u * NG * T;
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
    if (fl & (CSMC_DESC_INV | CSMC_DESC_EVAL)) return bounded_delay(n, rv.vars, rv.rates, li, lo, fl, x);
    const float inv = (fl & CSMC_DESC_PROG) ? rv.rates[lo] : __uint_as_float(lo);
    return exp_delay(x, inv);
}

// One component's part in the race: a class member updates its class's
// chain-k largest key, any other component (ALLCLS false) races with its own
// delay.  cb: 255 minus the component's bit-reversed index (bitrev_bits(cc,
// bits)), the low byte of its class key: (x | 0xff) - br = (x & ~0xff) | cb.
template <bool ALLCLS, uint32_t k>
static __device__ __forceinline__ void race_member(const Net &n, uint32_t bits, const CodedView &rv, uint32_t wd,
                                                   uint32_t cc, uint32_t x, uint32_t cb, unsigned long long &best,
                                                   float &bestd) {
    const uint32_t b = (wd >> (8u * k)) & 0xffu;
    const uint32_t code = b >> 5;
    const uint32_t T = rv.T;
    if (ALLCLS || code < CSMC_RACE_CLASSES) {
        const uint32_t key = (x & 0xffffff00u) | cb;
        uint32_t *pp = rv.keys + (code * 4u + k) * T;
        *pp = max(*pp, key);
    } else if (code == kCodeGeneral) {
        const float d = desc_delay(n, rv, n.comp[cc].loc_begin + (b & 31u), x);
        const unsigned long long key = (static_cast<unsigned long long>(delay_key(d)) << 32) | (255u - cb);
        if (key < best) {
            best = key;
            bestd = d;
        }
    }
}

// The race decided from the class keys (race_classes' decision over the
// same keys); false: the caller runs race_exact.  src: each class's 1/rate
// source (CSMC_CLASS_SRC_PROG | slot, or float bits).  ALLCLS: every
// location is classed, so no component takes the descriptor path.
template <bool ALLCLS>
static __device__ __forceinline__ bool race_coded(const Net &n, uint32_t C, uint32_t bits, uint32_t NG,
                                                  const CodedView &rv, const PhiloxKeys &K, const uint32_t *src,
                                                  uint64_t run, uint32_t step, unsigned long long &best,
                                                  float &bestd) {
    const uint32_t T = rv.T;
    for (uint32_t w = 0; w < 4u * NG; ++w) rv.keys[w * T] = 0u;
    best = ~0ull;
    bestd = 0.0f;
    const PhiloxStep ps = philox_step(K, step, run);
    // bit reversal of component 4q + k over `bits` (>= 2) bits: the two low
    // bits (k) become the top two, q the low bits - 2 reversed
    const uint32_t hi_shift = bits - 2u;  // bits >= 2: the plan needs at least four components
    const uint32_t Qf = C >> 2;           // words whose four components all exist
#pragma unroll kCodedUnroll
    for (uint32_t q = 0; q < Qf; ++q) {
        const u32x4 blk = philox_block(K, ps, q);
        const uint32_t wd = rv.lw[q * T], cc = 4u * q;
        const uint32_t rq = hi_shift ? (__brev(q) >> (32u - hi_shift)) : 0u;
        const uint32_t cb = 255u - rq;
        race_member<ALLCLS, 0>(n, bits, rv, wd, cc, blk.x, cb, best, bestd);
        race_member<ALLCLS, 1>(n, bits, rv, wd, cc + 1u, blk.y, cb - (2u << hi_shift), best, bestd);
        race_member<ALLCLS, 2>(n, bits, rv, wd, cc + 2u, blk.z, cb - (1u << hi_shift), best, bestd);
        race_member<ALLCLS, 3>(n, bits, rv, wd, cc + 3u, blk.w, cb - (3u << hi_shift), best, bestd);
    }
    if (C & 3u) {  // the last, partly filled word
        const u32x4 blk = philox_block(K, ps, Qf);
        const uint32_t wd = rv.lw[Qf * T], cc = 4u * Qf, rem = C & 3u;
        const uint32_t rq = hi_shift ? (__brev(Qf) >> (32u - hi_shift)) : 0u;
        const uint32_t cb = 255u - rq;
        race_member<ALLCLS, 0>(n, bits, rv, wd, cc, blk.x, cb, best, bestd);
        if (rem > 1u) race_member<ALLCLS, 1>(n, bits, rv, wd, cc + 1u, blk.y, cb - (2u << hi_shift), best, bestd);
        if (rem > 2u) race_member<ALLCLS, 2>(n, bits, rv, wd, cc + 2u, blk.z, cb - (1u << hi_shift), best, bestd);
    }
    // each class races with its largest key
    uint32_t inf_classes = 0, ties = 0;
    uint32_t top[CSMC_RACE_CLASSES];
    float dcls[CSMC_RACE_CLASSES], icls[CSMC_RACE_CLASSES];
#pragma unroll
    for (uint32_t g = 0; g < CSMC_RACE_CLASSES; ++g) {
        top[g] = 0u;
        dcls[g] = 0.0f;
        icls[g] = 0.0f;
        if (g >= NG) continue;
        const uint32_t *kg = rv.keys + (4u * g) * T;
        const uint32_t a = max(max(kg[0], kg[T]), max(kg[2u * T], kg[3u * T]));
        // key 0 (draw 0 at bit-reversed index 255) is also the "no member"
        // value; only component 255 of a 256-component network can hold it
        if (a == 0u && !(C == 256u && (rv.byte_of(255u) >> 5) == g)) continue;
        const uint32_t sg = src[g];
        const float inv = (sg & CSMC_CLASS_SRC_PROG) ? rv.rates[sg & 0xffffu] : __uint_as_float(sg);
        if (!(inv > 0.0f)) return false;  // delays 0, negative or NaN for the whole class
        if (!(inv <= 3.40282347e38f)) {   // +inf: the class's delays are +inf (NaN at u = 1)
            inf_classes |= 1u << g;
            continue;
        }
        const uint32_t m1 = a >> 8, br1 = 255u - (a & 255u);
        const float d1 = exp_delay(m1 << 8, inv);
        top[g] = a;
        dcls[g] = d1;
        icls[g] = inv;
        ties |= m1 > 0u ? (1u << g) : 0u;
        const unsigned long long key = (static_cast<unsigned long long>(delay_key(d1)) << 32) | br1;
        if (key < best) {
            best = key;
            bestd = d1;
        }
    }
    // a class can hide a tie (a lower draw of a member with a smaller index
    // that rounds to the same delay) only when its delay is the race's
    // minimum and its largest draw sits on a flat spot of the delay; the
    // exact race decides those steps
#pragma unroll
    for (uint32_t g = 0; g < CSMC_RACE_CLASSES; ++g) {
        if (!((ties >> g) & 1u) || dcls[g] != bestd) continue;
        if (exp_delay(((top[g] >> 8) - 1u) << 8, icls[g]) == dcls[g]) return false;
    }
    if (inf_classes && static_cast<uint32_t>(best >> 32) >= delay_key(__uint_as_float(0x7f800000u))) return false;
    return true;
}

#ifndef CSMC_CODED_MIN_CTAS_PER_SM
#define CSMC_CODED_MIN_CTAS_PER_SM 4
#endif

template <bool VERIFY, bool SLOTS, bool ALLCLS>
__global__ void __launch_bounds__(128, CSMC_CODED_MIN_CTAS_PER_SM) coded_kernel(const __grid_constant__ SimParams p) {
    extern __shared__ __align__(16) uint8_t smem[];
    stage_network(smem, p.blob, p.blob_bytes);
    const uint32_t C = p.net.n_comps, V = p.net.n_vars, P = p.net.n_rate_prog;
    const uint32_t T = blockDim.x, t = threadIdx.x;
    const bool recv = (p.net.recv_lo | p.net.recv_hi) != 0;
    const CodedView rv = carve_coded_view(smem + p.blob_bytes, V, P, C, p.net.n_classes, recv, T, t);
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
        if (!race_coded<ALLCLS>(n, C, bits, NG, rv, p.keys, p.class_src, run, step, best, bestd))
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

template <bool VERIFY, bool SLOTS, bool ALLCLS>
int coded_launch_one(const SimParams &p, int grid, int block, size_t smem, void *stream) {
    auto fn = detail::coded_kernel<VERIFY, SLOTS, ALLCLS>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool VERIFY, bool SLOTS, bool ALLCLS>
int coded_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::coded_kernel<VERIFY, SLOTS, ALLCLS>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
