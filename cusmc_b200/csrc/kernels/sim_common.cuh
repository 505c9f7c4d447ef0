// Device-side pieces shared by the two simulation kernel families
// (lane-group kernel: sim_impl.cuh; thread-per-run kernel: sim_serial.cuh).
// Semantics follow the reference kernel; file:line references are to
// simulation/simulation.cu and simulation/expressions.cu of the reference.
#pragma once
#include "sim.cuh"

#include <cuda_runtime.h>

namespace csmc {
namespace detail {

constexpr double kEps = 0.00001;                     // DBL_EPSILON, include/common_macros.h:72
constexpr double kDblMax = 1.7976931348623158e+308;  // include/common_macros.h:71
constexpr double kDblMin = 2.2250738585072014e-308;

// The packed network as seen from shared memory.
struct Net {
    const csmc_comp *comp;
    const csmc_loc *loc;
    const csmc_edge *edge;
    const csmc_guard *guard;
    const csmc_update *upd;
    const csmc_var *var;
    const double *konst;
    const uint64_t *code;
    const uint16_t *loc_rate;
    const float *inv_lit;
    const uint32_t *rate_prog;
    const uint16_t *clock;
    const uint64_t *loc_desc;
    const uint32_t *loc_inv1;  // CSMC_DESC_INV1 locations' invariant (null in blobs without the table)
    uint32_t n_comps, n_vars, n_rate_prog, flags, n_clocks, recv_lo, recv_hi;
};

static __device__ __forceinline__ Net net_view(const uint8_t *base) {
    const csmc_net_header *h = reinterpret_cast<const csmc_net_header *>(base);
    Net n;
    n.comp = reinterpret_cast<const csmc_comp *>(base + h->off_comp);
    n.loc = reinterpret_cast<const csmc_loc *>(base + h->off_loc);
    n.edge = reinterpret_cast<const csmc_edge *>(base + h->off_edge);
    n.guard = reinterpret_cast<const csmc_guard *>(base + h->off_guard);
    n.upd = reinterpret_cast<const csmc_update *>(base + h->off_update);
    n.var = reinterpret_cast<const csmc_var *>(base + h->off_var);
    n.konst = reinterpret_cast<const double *>(base + h->off_const);
    n.code = reinterpret_cast<const uint64_t *>(base + h->off_code);
    n.loc_rate = reinterpret_cast<const uint16_t *>(base + h->off_loc_rate);
    n.inv_lit = reinterpret_cast<const float *>(base + h->off_inv_lit);
    n.rate_prog = reinterpret_cast<const uint32_t *>(base + h->off_rate_prog);
    n.clock = reinterpret_cast<const uint16_t *>(base + h->off_clock);
    n.loc_desc = reinterpret_cast<const uint64_t *>(base + h->off_loc_desc);
    n.loc_inv1 = h->off_loc_inv1 ? reinterpret_cast<const uint32_t *>(base + h->off_loc_inv1) : nullptr;
    n.n_comps = h->n_comps;
    n.n_vars = h->n_vars;
    n.n_rate_prog = h->n_rate_prog;
    n.flags = h->flags;
    n.n_clocks = h->n_clocks;
    n.recv_lo = h->recv_chan_lo;
    n.recv_hi = h->recv_chan_hi;
    return n;
}

// The same view with offsets and counts taken from the kernel parameters.
static __device__ __forceinline__ Net net_view(const uint8_t *base, const NetLayout &l) {
    Net n;
    n.comp = reinterpret_cast<const csmc_comp *>(base + l.off_comp);
    n.loc = reinterpret_cast<const csmc_loc *>(base + l.off_loc);
    n.edge = reinterpret_cast<const csmc_edge *>(base + l.off_edge);
    n.guard = reinterpret_cast<const csmc_guard *>(base + l.off_guard);
    n.upd = reinterpret_cast<const csmc_update *>(base + l.off_update);
    n.var = reinterpret_cast<const csmc_var *>(base + l.off_var);
    n.konst = reinterpret_cast<const double *>(base + l.off_const);
    n.code = reinterpret_cast<const uint64_t *>(base + l.off_code);
    n.loc_rate = reinterpret_cast<const uint16_t *>(base + l.off_loc_rate);
    n.inv_lit = reinterpret_cast<const float *>(base + l.off_inv_lit);
    n.rate_prog = reinterpret_cast<const uint32_t *>(base + l.off_rate_prog);
    n.clock = reinterpret_cast<const uint16_t *>(base + l.off_clock);
    n.loc_desc = reinterpret_cast<const uint64_t *>(base + l.off_loc_desc);
    n.loc_inv1 = l.off_loc_inv1 ? reinterpret_cast<const uint32_t *>(base + l.off_loc_inv1) : nullptr;
    n.n_comps = l.n_comps;
    n.n_vars = l.n_vars;
    n.n_rate_prog = l.n_rate_prog;
    n.flags = l.flags;
    n.n_clocks = l.n_clocks;
    n.recv_lo = l.recv_lo;
    n.recv_hi = l.recv_hi;
    return n;
}

// Whether any location can receive on channel ch (> 0).
static __device__ __forceinline__ bool has_receivers(const Net &n, int ch) {
    if (ch < 32) return (n.recv_lo >> ch) & 1u;
    if (ch < 63) return (n.recv_hi >> (ch - 32)) & 1u;
    return (n.recv_hi >> 31) & 1u;
}

// A run's variables: element i at base[i * stride] (stride 1 for the
// lane-group kernel's shared array, the thread count for the thread-per-run
// kernel's interleaved arrays).
struct VarView {
    float *base;
    uint32_t stride;
    __device__ __forceinline__ float &operator[](uint32_t i) const { return base[i * stride]; }
};

static __device__ __forceinline__ void mix(unsigned long long &h, uint32_t w) { h = (h ^ w) * 0x100000001b3ull; }

// One operator of the expression language on the two top stack entries
// (v1 below v2); PN and tree operators (expressions.cu:88-173, 199-307).
static __device__ __forceinline__ double apply_op(uint32_t op, double v1, double v2) {
    switch (op) {
    case CSMC_OP_ADD: case CSMC_OP_TADD: return d_add(v1, v2);
    case CSMC_OP_SUB: case CSMC_OP_TSUB: return d_sub(v1, v2);
    case CSMC_OP_MUL: case CSMC_OP_TMUL: return d_mul(v1, v2);
    case CSMC_OP_DIV: return d_div(v1, v2);
    case CSMC_OP_TDIV: {
        if (v2 == 0.0) return 0.0;
        const double r = d_div(v1, v2);
        return r == 0.0 ? kDblMin : r;
    }
    case CSMC_OP_POW: return pow_model(v1, v2);
    case CSMC_OP_NEG: return -v2;
    case CSMC_OP_SQRT: return d_sqrt(v2);
    case CSMC_OP_MOD: {
        const int x = d2i_sat(v1), y = d2i_sat(d_add(v2, kEps));
        return (y == 0 || (x == (-2147483647 - 1) && y == -1)) ? 0.0 : static_cast<double>(x % y);
    }
    case CSMC_OP_AND: return (fabs(v1) > kEps && fabs(v2) > kEps) ? 1.0 : 0.0;
    case CSMC_OP_OR: return (fabs(v1) > kEps || fabs(v2) > kEps) ? 1.0 : 0.0;
    case CSMC_OP_LE: return v1 <= v2 ? 1.0 : 0.0;
    case CSMC_OP_GE: return v1 >= v2 ? 1.0 : 0.0;
    case CSMC_OP_LT: return v1 < v2 ? 1.0 : 0.0;
    case CSMC_OP_GT: return v1 > v2 ? 1.0 : 0.0;
    case CSMC_OP_EQ: return fabs(d_sub(v1, v2)) <= kEps ? 1.0 : 0.0;
    case CSMC_OP_NE: return fabs(d_sub(v1, v2)) > kEps ? 1.0 : 0.0;
    case CSMC_OP_NOT: return fabs(v2) < kEps ? 1.0 : 0.0;
    case CSMC_OP_RANDOM: return 1.0;
    case CSMC_OP_DUP: return v2;
    default: return 0.0;  // CSMC_OP_ZERO
    }
}

// General programs: a real stack.  PN operators push without popping
// (expressions.cu:192-193 pass stack_top by value); SKIP pops one; tree
// operators pop two.
static __device__ __noinline__ double eval_stack(const Net &n, VarView vars, uint32_t p) {
    double st[CSMC_MAX_STACK];
    int top = 0;
    for (uint32_t ip = p + 1;; ++ip) {
        const uint64_t ins = n.code[ip];
        const uint32_t op = CSMC_INS_OP(ins), a = CSMC_INS_A(ins);
        double r;
        if (op == CSMC_OP_END) return top > 0 ? st[top - 1] : 0.0;
        if (op == CSMC_OP_PUSH_C) r = n.konst[a];
        else if (op == CSMC_OP_PUSH_V) r = static_cast<double>(vars[a]);
        else if (op == CSMC_OP_SKIP) {
            --top;
            if (fabs(st[top]) > kEps) ip += a;
            continue;
        } else if (op >= CSMC_OP_TADD && op <= CSMC_OP_TDIV) {
            const double R = st[--top], L = st[--top];
            r = apply_op(op, L, R);
        } else {
            const double v2 = top >= 1 ? st[top - 1] : 0.0;
            const double v1 = top >= 2 ? st[top - 2] : 0.0;
            r = apply_op(op, v1, v2);
        }
        if (top < CSMC_MAX_STACK) st[top++] = r;
    }
}

// Programs that only ever read the two top entries (header flag WINDOW)
// run on two registers; the rest on the stack machine.
static __device__ __noinline__ double eval_prog(const Net &n, VarView vars, uint32_t p) {
    if (!(CSMC_INS_A(n.code[p]) & CSMC_PROG_WINDOW)) return eval_stack(n, vars, p);
    double a = 0.0, b = 0.0;
    for (uint32_t ip = p + 1;; ++ip) {
        const uint64_t ins = n.code[ip];
        const uint32_t op = CSMC_INS_OP(ins), x = CSMC_INS_A(ins);
        double r;
        if (op == CSMC_OP_END) return b;
        if (op == CSMC_OP_PUSH_C) r = n.konst[x];
        else if (op == CSMC_OP_PUSH_V) r = static_cast<double>(vars[x]);
        else r = apply_op(op, a, b);
        a = b;
        b = r;
    }
}

// Operand of a PUSH_C / PUSH_V instruction.
static __device__ __forceinline__ double chain_operand(const Net &n, VarView vars, uint64_t ins) {
    const uint32_t a = CSMC_INS_A(ins);
    return CSMC_INS_OP(ins) == CSMC_OP_PUSH_V ? static_cast<double>(vars[a]) : n.konst[a];
}

// v1 op v2 for the operators of CSMC_PROG_CHAIN programs (apply_op's
// arithmetic for them).
static __device__ __forceinline__ double chain_op(uint32_t op, double v1, double v2) {
    if (op == CSMC_OP_ADD || op == CSMC_OP_TADD) return d_add(v1, v2);
    if (op == CSMC_OP_SUB || op == CSMC_OP_TSUB) return d_sub(v1, v2);
    if (op == CSMC_OP_MUL || op == CSMC_OP_TMUL) return d_mul(v1, v2);
    return d_div(v1, v2);
}

// Any expression handle: literals and variables inline, programs of one or
// two binary operations (CSMC_PROG_CHAIN) inline, others out of line.
static __device__ __forceinline__ double eval(const Net &n, VarView vars, uint32_t h) {
    const uint32_t tag = CSMC_H_TAG(h), p = CSMC_H_PAYLOAD(h);
    if (tag == CSMC_H_LIT) return n.konst[p];
    if (tag == CSMC_H_VAR) return static_cast<double>(vars[p]);
    if (CSMC_INS_A(n.code[p]) & CSMC_PROG_CHAIN) {
        double r = chain_op(CSMC_INS_OP(n.code[p + 3]), chain_operand(n, vars, n.code[p + 1]),
                            chain_operand(n, vars, n.code[p + 2]));
        const uint64_t i4 = n.code[p + 4];
        if (CSMC_INS_OP(i4) != CSMC_OP_END) r = chain_op(CSMC_INS_OP(n.code[p + 5]), r, chain_operand(n, vars, i4));
        return r;
    }
    return eval_prog(n, vars, p);
}

// simulation.cu:184-266
static __device__ __forceinline__ bool guards_ok(const Net &n, VarView vars, const csmc_edge &e) {
    const uint32_t gb = CSMC_EDGE_GUARD_BEGIN(e), ng = CSMC_EDGE_N_GUARDS(e);
    for (uint32_t i = 0; i < ng; ++i) {
        const csmc_guard g = n.guard[gb + i];
        const double v = static_cast<double>(vars[g.var]);
        const double b = eval(n, vars, g.rhs);
        bool ok;
        switch (g.op) {
        case CSMC_G_LT: ok = v < b; break;
        case CSMC_G_LE: ok = v <= b; break;
        case CSMC_G_GT: ok = v > b; break;
        case CSMC_G_GE: ok = v >= b; break;
        case CSMC_G_EQ: ok = fabs(d_sub(v, b)) <= kEps; break;
        default: ok = false; break;
        }
        if (!ok) return false;
    }
    return true;
}

// Bound of the delay-bounding invariants of location L (simulation.cu:
// 461-511); returns false when no invariant bounds the delay.
static __device__ __forceinline__ bool delay_bound(const Net &n, VarView vars, const csmc_loc &L, double &max_delay) {
    max_delay = kDblMax;
    bool bounded = false;
    for (uint32_t i = 0; i < L.n_inv; ++i) {
        const csmc_guard g = n.guard[L.inv_begin + i];
        const double cur = static_cast<double>(vars[g.var]);
        const double bound = eval(n, vars, g.rhs);
        double ttb = d_sub(bound, cur);
        if (g.op == CSMC_G_LT) ttb = d_sub(ttb, 1e-6);
        if (ttb >= 0) {
            max_delay = fmin(max_delay, ttb);
            bounded = true;
        }
    }
    return bounded;
}

// simulation.cu:409-541 for one component in global location li; x is its
// delay draw; rates: the run's evaluated rate-program table.
static __device__ __forceinline__ float comp_delay(const Net &n, VarView vars, VarView rates, uint32_t li,
                                                   uint32_t x) {
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
    return exp_delay(x, inv);
}

// Delay of a CSMC_DESC_INV1 location (comp_delay's arithmetic for one
// invariant clock <= / < literal): uniform on (0, bound - clock] while the
// bound lies ahead, else exponential with the descriptor's 1/rate.
static __device__ __forceinline__ float inv1_delay(const Net &n, VarView vars, VarView rates, uint32_t li,
                                                   uint32_t lo, uint32_t fl, uint32_t x) {
    const uint32_t w = n.loc_inv1[li];
    double ttb = d_sub(n.konst[CSMC_INV1_CONST(w)], static_cast<double>(vars[CSMC_INV1_VAR(w)]));
    if (CSMC_INV1_STRICT(w)) ttb = d_sub(ttb, 1e-6);
    if (ttb >= 0) return uniform_delay(x, ttb);
    return exp_delay(x, (fl & CSMC_DESC_PROG) ? rates[lo] : __uint_as_float(lo));
}

// Enabled-edge slot state after writing the enabled list `en` (ascending):
// slot j holds edge j exactly when edges 0..j are all enabled.
static __device__ __forceinline__ uint32_t write_slots(uint32_t mask, uint32_t en) {
    const uint32_t cnt = __popc(en);
    if (cnt == 0) return mask;
    const uint32_t p = static_cast<uint32_t>(__ffs(~en) ? __ffs(~en) - 1 : 32);  // trailing ones
    const uint32_t low_n = cnt >= 32 ? 0xffffffffu : ((1u << cnt) - 1u);
    const uint32_t low_p = p >= 32 ? 0xffffffffu : ((1u << p) - 1u);
    return (mask & ~low_n) | low_p;
}

static __device__ __forceinline__ uint32_t nth_bit(uint32_t m, uint32_t k) {  // index of the k-th set bit
    for (uint32_t i = 0; i < k; ++i) m &= m - 1;
    return static_cast<uint32_t>(__ffs(m) - 1);
}

// Scalars of one run (the reference's SharedBlockMemory fields besides the
// variables, simulation/state/shared_run_state.cuh:26-48).
struct RunScalars {
    double qmin, qmax;
    unsigned long long digest;
    int chan, sender, goal, pad;
};

// simulation.cu:9-24 + 27-181: choose among the enabled edges `en` of
// component c in local location cur_loc and apply the chosen edge.  Returns
// the new local location.
template <bool VERIFY, class S>
static __device__ __forceinline__ uint32_t take_edge(const Net &n, VarView vars, S &st, uint64_t seed,
                                                     int32_t var_id, uint64_t run, uint32_t step, uint32_t c,
                                                     uint32_t cur_loc, uint32_t en, uint32_t slot_mask,
                                                     uint32_t which) {
    const csmc_loc L = n.loc[n.comp[c].loc_begin + cur_loc];
    const uint32_t cnt = __popc(en);
    uint32_t sel = static_cast<uint32_t>(__ffs(en) - 1);
    if (cnt > 1) {
        double sum = 0.0;
        for (uint32_t i = 0; i < L.n_edges; ++i)
            if ((slot_mask >> i) & 1u) sum = d_add(sum, eval(n, vars, n.edge[L.edge_begin + i].weight));
        const int W = d2i_sat(sum);
        const float u = uniform01(choice_word(seed, run, step, c, which));
        const int rnd = f2i_sat(f_mul(static_cast<float>(W), u));
        uint32_t temp = static_cast<uint32_t>(W);
        for (int i = static_cast<int>(cnt) - 1; i >= 0; --i) {
            const int w = d2i_sat(eval(n, vars, n.edge[L.edge_begin + i].weight));
            if (static_cast<int>(temp - static_cast<uint32_t>(w)) <= rnd) {
                sel = nth_bit(en, static_cast<uint32_t>(i));
                break;
            }
            temp -= static_cast<uint32_t>(w);
        }
    }
    if (VERIFY) mix(st.digest, sel);
    const csmc_edge e = n.edge[L.edge_begin + sel];
    if (e.channel > 0) {
        st.chan = e.channel;
        st.sender = static_cast<int>(c);
    }
    const uint32_t ub = CSMC_EDGE_UPD_BEGIN(e), nu = CSMC_EDGE_N_UPD(e);
    for (uint32_t i = 0; i < nu; ++i) {
        const csmc_update u = n.upd[ub + i];
        const double nv = eval(n, vars, u.expr);
        if (static_cast<int32_t>(u.var) == var_id) {
            if (nv > st.qmax) st.qmax = nv;
            if (nv < st.qmin) st.qmin = nv;
        }
        vars[u.var] = d2f(nv);
        if (VERIFY) {
            mix(st.digest, u.var);
            mix(st.digest, f_bits(vars[u.var]));
        }
    }
    if (e.dst_local < 0) return cur_loc;
    const uint32_t dst = static_cast<uint32_t>(e.dst_local);
    if (n.loc[n.comp[c].loc_begin + dst].type == CSMC_GOAL) st.goal = 1;
    return dst;
}

// Enabled non-receiving edges of a location (simulation.cu:268-305).
static __device__ __forceinline__ uint32_t enabled_edges(const Net &n, VarView vars, uint32_t li) {
    const csmc_loc L = n.loc[li];
    uint32_t en = 0;
    for (uint32_t i = 0; i < L.n_edges; ++i) {
        const csmc_edge e = n.edge[L.edge_begin + i];
        if (e.channel >= 0 && guards_ok(n, vars, e)) en |= 1u << i;
    }
    return en;
}

// Enabled receiving edges on channel chan (SyncInSerial's parallel phase,
// simulation.cu:363-377).
static __device__ __forceinline__ uint32_t recv_edges(const Net &n, VarView vars, uint32_t li, int chan) {
    const csmc_loc L = n.loc[li];
    uint32_t m = 0;
    for (uint32_t i = 0; i < L.n_edges; ++i) {
        const csmc_edge e = n.edge[L.edge_begin + i];
        if (e.channel == -chan && guards_ok(n, vars, e)) m |= 1u << i;
    }
    return m;
}

static __device__ __forceinline__ void stage_network(uint8_t *smem, const uint8_t *blob, uint32_t bytes) {
    const int4 *src = reinterpret_cast<const int4 *>(blob);
    int4 *dst = reinterpret_cast<int4 *>(smem);
    for (uint32_t i = threadIdx.x; i < bytes / 16; i += blockDim.x) dst[i] = src[i];
}

}  // namespace detail
}  // namespace csmc
