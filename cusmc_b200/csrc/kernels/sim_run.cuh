// One run owned by one thread: the state layout and the step of the
// thread-per-run kernels (the single-network kernel of sim_serial.cuh and
// the multi-network batch kernel of sim_batch.cuh share these, force-inlined).
//
// Per-run state lives in interleaved arrays (element i of thread t at
// [i * T + t]; conflict-free in shared memory, coalesced in global memory):
// variables, the evaluated rate table, a snapshot of the variables for
// broadcast receivers, component locations and, when some location has
// several edges, the enabled-edge slot masks.
//
// The component order, the race tie-break, the Philox draws and every
// arithmetic step follow the reference kernel (simulation/simulation.cu:
// 674-901) and are those of the lane-group kernel and the CPU oracle.
#pragma once
#include "sim_common.cuh"

namespace csmc {
namespace detail {

// Delay of a component whose descriptor flags INV or EVAL: the one-
// invariant form inline here, the rest through comp_delay.  One call site
// per component keeps the race loops' register budget.
static __device__ __noinline__ float bounded_delay(const Net &n, VarView vars, VarView rates, uint32_t li,
                                                   uint32_t lo, uint32_t fl, uint32_t x) {
    if (fl & CSMC_DESC_INV1) return inv1_delay(n, vars, rates, li, lo, fl, x);
    return comp_delay(n, vars, rates, li, x);
}

template <bool LOC8>
struct LocStore {
    using T = uint16_t;  // global location index
};
template <>
struct LocStore<true> {
    using T = uint8_t;  // local location index
};

// Views of one thread's run state.  LOC8: locations stored as 8-bit local
// indices (automata of at most 256 locations), else 16-bit global indices.
template <bool LOC8>
struct RunView {
    using LocT = typename LocStore<LOC8>::T;
    VarView vars, rates, shadow;
    LocT *locs;       // this thread's element 0; stride T
    uint32_t *slotv;  // this thread's element 0; stride T
    uint32_t *cls;    // race-class keys: [g] largest, [4 + g] second largest; stride T
    uint32_t T;

    // global location index of component c
    __device__ __forceinline__ uint32_t loc(const Net &n, uint32_t c) const {
        return LOC8 ? n.comp[c].loc_begin + locs[c * T] : locs[c * T];
    }
    __device__ __forceinline__ void set_local(const Net &n, uint32_t c, uint32_t local) const {
        locs[c * T] = static_cast<LocT>(LOC8 ? local : n.comp[c].loc_begin + local);
    }
};

// Bytes of one thread's run state with V variables, P rate programs and C
// components (the layout carve_run_view uses).
static __host__ __device__ __forceinline__ uint32_t run_loc_bytes(uint32_t C, uint32_t T, bool loc8) {
    return loc8 ? ((C * T + 3u) & ~3u) : ((2u * C * T + 3u) & ~3u);
}

// Carves thread t's views out of a state slab of T threads laid out as
// vars[V] | rates[P] | shadow[V] (floats) | race-class keys[8] | locs[C] |
// slots[C] (u32).
template <bool LOC8>
static __device__ __forceinline__ RunView<LOC8> carve_run_view(uint8_t *st, uint32_t V, uint32_t P, uint32_t C,
                                                                 uint32_t T, uint32_t t) {
    using LocT = typename LocStore<LOC8>::T;
    float *fb = reinterpret_cast<float *>(st);
    RunView<LOC8> r;
    r.vars = VarView{fb + t, T};
    r.rates = VarView{fb + V * T + t, T};
    r.shadow = VarView{fb + (V + P) * T + t, T};
    r.cls = reinterpret_cast<uint32_t *>(st + 4u * (2u * V + P) * T) + t;
    const uint32_t lb = 4u * (2u * V + P + 2u * CSMC_RACE_CLASSES) * T;
    r.locs = reinterpret_cast<LocT *>(st + lb) + t;
    r.slotv = reinterpret_cast<uint32_t *>(st + lb + run_loc_bytes(C, T, LOC8)) + t;
    r.T = T;
    return r;
}

// Run initialisation (simulation.cu:766-831): initial locations, slot
// masks, initial variable values, query extremes.
template <bool SLOTS, class RV>
static __device__ __forceinline__ void run_init(const Net &n, uint32_t C, uint32_t V, const RV &rv,
                                                RunScalars &sc, int var_id) {
    for (uint32_t c = 0; c < C; ++c) {
        rv.set_local(n, c, n.comp[c].init_local);
        if (SLOTS) rv.slotv[c * rv.T] = 0u;
    }
    for (uint32_t v = 0; v < V; ++v) rv.vars[v] = n.var[v].init;
    double q0 = 0.0;
    if (var_id >= 0 && static_cast<uint32_t>(var_id) < V && n.var[var_id].kind == 0)
        q0 = static_cast<double>(n.var[var_id].init);
    sc = RunScalars{q0, q0, 0xcbf29ce484222325ull, 0, -1, 0, 0};
}

// Per-run outcome at the end of a run (simulation.cu:835-849, 887-893).
struct RunEnd {
    bool done;
    uint32_t flag, capped;
    double value;
};

static __device__ __forceinline__ RunEnd run_end(const RunScalars &sc, float time, float horizon, uint32_t step,
                                                 uint64_t cap, int loc_mode, int is_max, double threshold) {
    RunEnd r;
    const bool timeout = !(time < horizon);
    const bool at_goal = loc_mode && sc.goal;
    const bool at_cap = step >= cap;
    r.done = timeout || at_goal || at_cap;
    r.capped = (!timeout && !at_goal && at_cap) ? 1u : 0u;
    r.value = is_max ? sc.qmax : sc.qmin;
    r.flag = (!timeout && at_goal) ? 1u : 0u;
    if (!loc_mode) r.flag = is_max ? (r.value > threshold) : (r.value < threshold);
    return r;
}

// Final state for verification: local locations, then variable bits.
template <class RV>
static __device__ __forceinline__ void run_final_state(const Net &n, uint32_t C, uint32_t V, const RV &rv,
                                                       uint32_t *w) {
    for (uint32_t c = 0; c < C; ++c) w[c] = rv.loc(n, c) - n.comp[c].loc_begin;
    for (uint32_t v = 0; v < V; ++v) w[C + v] = f_bits(rv.vars[v]);
}

// Pending broadcast receivers of the previous step's sender (SyncInSerial,
// simulation.cu:357-407): enabled sets from the state the sender left (the
// snapshot), then transitions in component order on the live state.
// Returns true when a receiver took an edge.
template <bool VERIFY, bool SLOTS, class RV>
static __device__ __forceinline__ bool run_receivers(const Net &n, uint32_t C, uint32_t V, const RV &rv,
                                                     RunScalars &sc, uint64_t seed, int var_id, uint64_t run,
                                                     uint32_t step) {
    if (sc.chan <= 0) return false;
    const uint32_t T = rv.T;
    const int chan = sc.chan, sender = sc.sender;
    bool moved = false;
    if (has_receivers(n, chan)) {
        for (uint32_t v = 0; v < V; ++v) rv.shadow[v] = rv.vars[v];
        for (uint32_t c = 0; c < C; ++c) {
            if (static_cast<int>(c) == sender) continue;
            const uint32_t li = rv.loc(n, c);
            if (!n.loc[li].n_recv) continue;
            const uint32_t m = recv_edges(n, rv.shadow, li, chan);
            if (!m) continue;
            uint32_t sm = 0;
            if (SLOTS) {
                sm = write_slots(rv.slotv[c * T], m);
                rv.slotv[c * T] = sm;
            }
            if (VERIFY) mix(sc.digest, c | 0x80000000u);
            const uint32_t base = n.comp[c].loc_begin;
            const uint32_t nl = take_edge<VERIFY>(n, rv.vars, sc, seed, var_id, run, step, c, li - base, m, sm, 1);
            rv.set_local(n, c, nl);
            moved = true;
        }
    }
    sc.chan = 0;
    sc.sender = -1;
    return moved;
}

// The race's outcome applied (simulation.cu:632-667, 876-882): clocks
// advance by dmin, the winner takes an enabled edge, time advances.
// Returns true when the winner took an edge.
template <bool VERIFY, bool SLOTS, class RV>
static __device__ __forceinline__ bool run_commit(const Net &n, uint32_t n_clocks, const RV &rv,
                                                  RunScalars &sc, uint64_t seed, int var_id, uint64_t run,
                                                  uint32_t &step, float &time, uint32_t win, float dmin) {
    const uint32_t T = rv.T;
    const VarView vars = rv.vars;
    bool took = false;
    if (VERIFY) {
        mix(sc.digest, step);
        mix(sc.digest, win);
        mix(sc.digest, f_bits(dmin));
    }
    if (static_cast<double>(dmin) < kDblMax) {
        for (uint32_t j = 0; j < n_clocks; ++j) {
            const uint32_t v = n.clock[j];
            vars[v] = d2f(d_add(static_cast<double>(vars[v]), static_cast<double>(dmin)));
        }
        const uint32_t li = rv.loc(n, win);
        const uint32_t en = enabled_edges(n, vars, li);
        uint32_t sm = 0;
        if (SLOTS) {
            sm = write_slots(rv.slotv[win * T], en);
            rv.slotv[win * T] = sm;
        }
        if (en) {
            const uint32_t base = n.comp[win].loc_begin;
            const uint32_t nl = take_edge<VERIFY>(n, vars, sc, seed, var_id, run, step, win, li - base, en, sm, 0);
            rv.set_local(n, win, nl);
            took = true;
        } else if (VERIFY) {
            mix(sc.digest, 0xffffffffu);
        }
    }
    time = d2f(d_add(static_cast<double>(time), static_cast<double>(dmin)));
    ++step;
    return took;
}

// The race over every component (simulation.cu:409-628): per-component
// delays, minimum of (delay key, bit-reversed index).
template <class RV>
static __device__ __forceinline__ void race_exact(const Net &n, uint32_t C, uint32_t bits, const RV &rv,
                                                  uint64_t seed, uint64_t run, uint32_t step, unsigned long long &best,
                                                  float &bestd) {
    best = ~0ull;
    bestd = 0.0f;
    for (uint32_t c = 0; c < C; c += 4) {
        const u32x4 blk = delay_block(seed, run, step, c >> 2);
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t cc = c + k;
            if (cc < C) {
                // fast path from the location's delay descriptor: the
                // exponential delay with the literal 1/rate or the step's
                // evaluated rate; zero-delay types and bounded locations
                // take the general path
                const uint32_t li = rv.loc(n, cc);
                const uint64_t dsc = n.loc_desc[li];
                const uint32_t lo = static_cast<uint32_t>(dsc), fl = static_cast<uint32_t>(dsc >> 32);
                const uint32_t x = word_of(blk, k);
                float inv = __uint_as_float(lo);
                if (fl & CSMC_DESC_PROG) inv = rv.rates[lo];
                float d = exp_delay(x, inv);
                if (fl & (CSMC_DESC_ZERO | CSMC_DESC_INV | CSMC_DESC_EVAL))
                    d = (fl & CSMC_DESC_ZERO) ? 0.0f : bounded_delay(n, rv.vars, rv.rates, li, lo, fl, x);
                const unsigned long long key =
                    (static_cast<unsigned long long>(delay_key(d)) << 32) | bitrev_bits(cc, bits);
                if (key < best) {
                    best = key;
                    bestd = d;
                }
            }
        }
    }
}

// The same race decided from race classes: within a class the delay is a
// non-increasing function of the 24-bit uniform draw m (log2 of the draw is
// monotone over all 2^24 draws, and multiplying by a positive 1/rate keeps
// the order), so a class is represented by its largest key (m, then the
// smallest bit-reversed index) and needs no logarithm per member.  Two
// members of a class tie only when their draws give the same float delay;
// when that cannot be ruled out from the two largest keys (or when a class's
// 1/rate is not finite and positive and the class could take part in the
// minimum) the function returns false and the caller runs race_exact.
template <class RV>
static __device__ __forceinline__ bool race_classes(const Net &n, uint32_t C, uint32_t bits, const RV &rv,
                                                    uint64_t seed, uint64_t run, uint32_t step,
                                                    unsigned long long &best, float &bestd) {
    const uint32_t T = rv.T;
    uint32_t pres = 0, pres2 = 0;
    best = ~0ull;
    bestd = 0.0f;
    for (uint32_t c = 0; c < C; c += 4) {
        const u32x4 blk = delay_block(seed, run, step, c >> 2);
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t cc = c + k;
            if (cc < C) {
                const uint32_t li = rv.loc(n, cc);
                const uint64_t dsc = n.loc_desc[li];
                const uint32_t lo = static_cast<uint32_t>(dsc), fl = static_cast<uint32_t>(dsc >> 32);
                const uint32_t x = word_of(blk, k);
                const uint32_t br = bitrev_bits(cc, bits);
                const uint32_t g = CSMC_DESC_CLASS(fl);
                if (g < CSMC_RACE_CLASSES) {
                    // branch-free update of the class's two largest keys
                    // (slots of absent classes hold stale values; the
                    // presence bits decide)
                    const uint32_t key = (x & 0xffffff00u) | (255u - br);
                    const uint32_t bit = 1u << g;
                    uint32_t *k1 = rv.cls + g * T, *k2 = rv.cls + (CSMC_RACE_CLASSES + g) * T;
                    const uint32_t a = *k1, b = *k2;
                    const bool p1 = (pres & bit) != 0, p2 = (pres2 & bit) != 0;
                    const bool gt1 = !p1 || key > a;
                    *k1 = gt1 ? key : a;
                    *k2 = gt1 ? (p1 ? a : b) : ((!p2 || key > b) ? key : b);
                    pres2 |= pres & bit;
                    pres |= bit;
                } else {
                    float d;
                    if (fl & CSMC_DESC_ZERO) {
                        d = 0.0f;
                    } else if (fl & (CSMC_DESC_INV | CSMC_DESC_EVAL)) {
                        d = bounded_delay(n, rv.vars, rv.rates, li, lo, fl, x);
                    } else {
                        const float inv = (fl & CSMC_DESC_PROG) ? rv.rates[lo] : __uint_as_float(lo);
                        d = exp_delay(x, inv);
                    }
                    const unsigned long long key = (static_cast<unsigned long long>(delay_key(d)) << 32) | br;
                    if (key < best) {
                        best = key;
                        bestd = d;
                    }
                }
            }
        }
    }
    uint32_t inf_classes = 0;
#pragma unroll
    for (uint32_t g = 0; g < CSMC_RACE_CLASSES; ++g) {
        const uint32_t bit = 1u << g;
        if (!(pres & bit)) continue;
        const uint32_t a = rv.cls[g * T];
        const uint32_t m1 = a >> 8, br1 = 255u - (a & 255u);
        const uint32_t li = rv.loc(n, bitrev_bits(br1, bits));
        const uint64_t dsc = n.loc_desc[li];
        const uint32_t lo = static_cast<uint32_t>(dsc), fl = static_cast<uint32_t>(dsc >> 32);
        const float inv = (fl & CSMC_DESC_PROG) ? rv.rates[lo] : __uint_as_float(lo);
        if (!(inv > 0.0f)) return false;  // delays 0, negative or NaN for the whole class
        if (!(inv <= 3.40282347e38f)) {   // +inf: the class's delays are +inf (NaN at u = 1)
            inf_classes |= bit;
            continue;
        }
        const float d1 = exp_delay(m1 << 8, inv);
        if (m1 > 0 && (pres2 & bit) && exp_delay((m1 - 1u) << 8, inv) == d1) {
            const uint32_t m2 = rv.cls[(CSMC_RACE_CLASSES + g) * T] >> 8;
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

// One step of a run: pending broadcast receivers, the per-step rate table,
// the race, the clock advance and the winner's transition, the time update.
// CLASSES: the network's descriptors carry race classes (C <= 256).
template <bool VERIFY, bool SLOTS, bool CLASSES, class RV>
static __device__ __forceinline__ void run_step(const Net &n, uint32_t C, uint32_t V, uint32_t P, uint32_t n_clocks,
                                                bool rate_table, const RV &rv, RunScalars &sc,
                                                uint64_t seed, int var_id, uint64_t run, uint32_t &step,
                                                float &time) {
    const uint32_t bits = ceil_log2(C);
    run_receivers<VERIFY, SLOTS>(n, C, V, rv, sc, seed, var_id, run, step);

    // ---- distinct rate programs, once per step
    if (rate_table)
        for (uint32_t j = 0; j < P; ++j) rv.rates[j] = inv_rate(eval(n, rv.vars, n.rate_prog[j]));

    // ---- delays and the race
    unsigned long long best;
    float bestd;
    if (CLASSES) {
        if (!race_classes(n, C, bits, rv, seed, run, step, best, bestd))
            race_exact(n, C, bits, rv, seed, run, step, best, bestd);
    } else {
        race_exact(n, C, bits, rv, seed, run, step, best, bestd);
    }
    const uint32_t win = bitrev_bits(static_cast<uint32_t>(best & 0xffffffffull), bits);
    run_commit<VERIFY, SLOTS>(n, n_clocks, rv, sc, seed, var_id, run, step, time, win, bestd);
}

}  // namespace detail
}  // namespace csmc
