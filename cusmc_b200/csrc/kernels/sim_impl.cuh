// Simulation kernel template (see sim.cuh for the mapping); instantiated
// per (lanes per run, components per lane) shape in sim_shapes_*.cu.
// Semantics follow the reference kernel line by line; file:line references
// are to simulation/simulation.cu and simulation/expressions.cu of the
// reference.
#pragma once
#include "sim.cuh"

#include <cuda_runtime.h>

namespace csmc {
namespace detail {

constexpr double kEps = 0.00001;                     // DBL_EPSILON, include/common_macros.h:72
constexpr double kDblMax = 1.7976931348623158e+308;  // include/common_macros.h:71
constexpr double kDblMin = 2.2250738585072014e-308;

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
    uint32_t n_comps, n_vars, n_rate_prog, flags;
};

struct RunState {  // per group, in shared memory
    double qmin, qmax;
    unsigned long long digest;
    int chan, sender, goal, pad;
    uint32_t pad2[2];
    float vars[1];  // n_vars entries, then n_rate_prog inverse rates
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
static __device__ __noinline__ double eval_stack(const Net &n, const float *vars, uint32_t p) {
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

// Any expression handle.  Literals and variables directly; programs that
// only ever read the two top entries (header flag WINDOW) with two
// registers; the rest on the stack machine.
static __device__ __forceinline__ double eval(const Net &n, const float *vars, uint32_t h) {
    const uint32_t tag = CSMC_H_TAG(h), p = CSMC_H_PAYLOAD(h);
    if (tag == CSMC_H_LIT) return n.konst[p];
    if (tag == CSMC_H_VAR) return static_cast<double>(vars[p]);
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

// simulation.cu:184-266
static __device__ __noinline__ bool guards_ok(const Net &n, const float *vars, const csmc_edge &e) {
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

// simulation.cu:409-541 for one component in location li; x is its delay draw.
static __device__ __forceinline__ float comp_delay(const Net &n, const RunState *s, uint32_t li, uint32_t x) {
    const csmc_loc L = n.loc[li];
    if (L.type > 1) return 0.0f;
    if (L.n_inv) {
        double max_delay = kDblMax;
        bool bounded = false;
        for (uint32_t i = 0; i < L.n_inv; ++i) {
            const csmc_guard g = n.guard[L.inv_begin + i];
            const double cur = static_cast<double>(s->vars[g.var]);
            const double bound = eval(n, s->vars, g.rhs);
            double ttb = d_sub(bound, cur);
            if (g.op == CSMC_G_LT) ttb = d_sub(ttb, 1e-6);
            if (ttb >= 0) {
                max_delay = fmin(max_delay, ttb);
                bounded = true;
            }
        }
        if (bounded) return uniform_delay(x, max_delay);
    }
    float inv;
    if (n.flags & CSMC_NET_RATE_TABLE) {
        const uint32_t slot = n.loc_rate[li];
        inv = (slot & CSMC_RATE_PROG_BIT) ? s->vars[n.n_vars + (slot & ~CSMC_RATE_PROG_BIT)] : n.inv_lit[slot];
    } else {
        inv = inv_rate(eval(n, s->vars, L.rate));
    }
    return exp_delay(x, inv);
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

// simulation.cu:9-24 + 27-181: choose among the enabled edges `en` of
// component c (location L), apply the edge.  Returns the new local location.
template <bool VERIFY>
static __device__ __noinline__ uint32_t take(const Net &n, RunState *s, const SimParams &p, uint64_t run,
                                             uint32_t step, uint32_t c, uint32_t cur_loc, uint32_t en,
                                             uint32_t slot_mask, uint32_t which) {
    const csmc_loc L = n.loc[n.comp[c].loc_begin + cur_loc];
    const uint32_t cnt = __popc(en);
    uint32_t sel = static_cast<uint32_t>(__ffs(en) - 1);
    if (cnt > 1) {
        double sum = 0.0;
        for (uint32_t i = 0; i < L.n_edges; ++i)
            if ((slot_mask >> i) & 1u) sum = d_add(sum, eval(n, s->vars, n.edge[L.edge_begin + i].weight));
        const int W = d2i_sat(sum);
        const float u = uniform01(choice_word(p.seed, run, step, c, which));
        const int rnd = f2i_sat(f_mul(static_cast<float>(W), u));
        uint32_t temp = static_cast<uint32_t>(W);
        for (int i = static_cast<int>(cnt) - 1; i >= 0; --i) {
            const int w = d2i_sat(eval(n, s->vars, n.edge[L.edge_begin + i].weight));
            if (static_cast<int>(temp - static_cast<uint32_t>(w)) <= rnd) {
                sel = nth_bit(en, static_cast<uint32_t>(i));
                break;
            }
            temp -= static_cast<uint32_t>(w);
        }
    }
    if (VERIFY) mix(s->digest, sel);
    const csmc_edge e = n.edge[L.edge_begin + sel];
    if (e.channel > 0) {
        s->chan = e.channel;
        s->sender = static_cast<int>(c);
    }
    const uint32_t ub = CSMC_EDGE_UPD_BEGIN(e), nu = CSMC_EDGE_N_UPD(e);
    for (uint32_t i = 0; i < nu; ++i) {
        const csmc_update u = n.upd[ub + i];
        const double nv = eval(n, s->vars, u.expr);
        if (static_cast<int32_t>(u.var) == p.var_id) {
            if (nv > s->qmax) s->qmax = nv;
            if (nv < s->qmin) s->qmin = nv;
        }
        s->vars[u.var] = d2f(nv);
        if (VERIFY) {
            mix(s->digest, u.var);
            mix(s->digest, f_bits(s->vars[u.var]));
        }
    }
    if (e.dst_local < 0) return cur_loc;
    const uint32_t dst = static_cast<uint32_t>(e.dst_local);
    if (n.loc[n.comp[c].loc_begin + dst].type == CSMC_GOAL) s->goal = 1;
    return dst;
}

// The winner's step (simulation.cu:656-667): enabled edges, slot update,
// transition.  Returns the new location; *slots is updated.
template <bool VERIFY>
static __device__ __noinline__ uint32_t win_step(const Net &n, RunState *s, const SimParams &p, uint64_t run,
                                                 uint32_t step, uint32_t c, uint32_t cur_loc, uint32_t *slots) {
    const csmc_loc L = n.loc[n.comp[c].loc_begin + cur_loc];
    uint32_t en = 0;
    for (uint32_t i = 0; i < L.n_edges; ++i) {
        const csmc_edge e = n.edge[L.edge_begin + i];
        if (e.channel >= 0 && guards_ok(n, s->vars, e)) en |= 1u << i;
    }
    *slots = write_slots(*slots, en);
    if (en) return take<VERIFY>(n, s, p, run, step, c, cur_loc, en, *slots, 0);
    if (VERIFY) mix(s->digest, 0xffffffffu);
    return cur_loc;
}

// Enabled receiving edges of component c in its location (SyncInSerial's
// parallel phase, simulation.cu:363-377).
static __device__ __noinline__ uint32_t recv_mask(const Net &n, const RunState *s, uint32_t li, int chan) {
    const csmc_loc L = n.loc[li];
    uint32_t m = 0;
    for (uint32_t i = 0; i < L.n_edges; ++i) {
        const csmc_edge e = n.edge[L.edge_begin + i];
        if (e.channel == -chan && guards_ok(n, s->vars, e)) m |= 1u << i;
    }
    return m;
}

#ifndef CSMC_MIN_CTAS_PER_SM
#define CSMC_MIN_CTAS_PER_SM 2
#endif

template <int G, int K, bool VERIFY>
__global__ void __launch_bounds__(256, CSMC_MIN_CTAS_PER_SM) sim_kernel(const SimParams p) {
    extern __shared__ __align__(16) uint8_t smem[];
    {  // stage the packed network (16-byte copies)
        const int4 *src = reinterpret_cast<const int4 *>(p.blob);
        int4 *dst = reinterpret_cast<int4 *>(smem);
        for (uint32_t i = threadIdx.x; i < p.blob_bytes / 16; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const csmc_net_header *h = reinterpret_cast<const csmc_net_header *>(smem);
    Net n;
    n.comp = reinterpret_cast<const csmc_comp *>(smem + h->off_comp);
    n.loc = reinterpret_cast<const csmc_loc *>(smem + h->off_loc);
    n.edge = reinterpret_cast<const csmc_edge *>(smem + h->off_edge);
    n.guard = reinterpret_cast<const csmc_guard *>(smem + h->off_guard);
    n.upd = reinterpret_cast<const csmc_update *>(smem + h->off_update);
    n.var = reinterpret_cast<const csmc_var *>(smem + h->off_var);
    n.konst = reinterpret_cast<const double *>(smem + h->off_const);
    n.code = reinterpret_cast<const uint64_t *>(smem + h->off_code);
    n.loc_rate = reinterpret_cast<const uint16_t *>(smem + h->off_loc_rate);
    n.inv_lit = reinterpret_cast<const float *>(smem + h->off_inv_lit);
    n.rate_prog = reinterpret_cast<const uint32_t *>(smem + h->off_rate_prog);
    n.n_comps = h->n_comps;
    n.n_vars = h->n_vars;
    n.n_rate_prog = h->n_rate_prog;
    n.flags = h->flags;
    const uint32_t C = n.n_comps, V = n.n_vars;
    const uint32_t bits = ceil_log2(C);
    const bool rate_table = (n.flags & CSMC_NET_RATE_TABLE) && n.n_rate_prog > 0;

    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gl = lane % G;  // lane within group
    const uint32_t gbase = lane - gl;
    const uint32_t gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << gbase);
    RunState *s = reinterpret_cast<RunState *>(smem + p.blob_bytes + (threadIdx.x / G) * p.state_stride);
    const uint32_t c0 = gl * K;

    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;
    const float T = p.horizon;
    const uint64_t cap = p.max_steps;

    for (;;) {
        unsigned long long ridx = 0;
        if (gl == 0) ridx = atomicAdd(p.scratch, 1ull);
        ridx = __shfl_sync(gmask, ridx, 0, G);
        if (ridx >= p.n_runs) break;
        const uint64_t run = p.first_run + ridx;

        // run initialisation (simulation.cu:766-831)
        for (uint32_t v = gl; v < V; v += G) s->vars[v] = n.var[v].init;
        if (gl == 0) {
            double q0 = 0.0;
            if (p.var_id >= 0 && static_cast<uint32_t>(p.var_id) < V && n.var[p.var_id].kind == 0)
                q0 = static_cast<double>(n.var[p.var_id].init);
            s->qmin = q0;
            s->qmax = q0;
            s->chan = 0;
            s->sender = -1;
            s->goal = 0;
            s->digest = 0xcbf29ce484222325ull;
        }
        uint32_t loc[K], slots[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint32_t c = c0 + k;
            loc[k] = c < C ? n.comp[c].loc_begin + n.comp[c].init_local : 0u;  // global location index
            slots[k] = 0u;
        }
        __syncwarp(gmask);

        float time = 0.0f;
        uint32_t step = 0;
        uint32_t flag = 0, capped = 0;
        while (time < T) {  // simulation.cu:835
            if (p.loc_mode && s->goal) {  // simulation.cu:839-849
                flag = 1;
                break;
            }
            if (step >= cap) {
                capped = 1;
                break;
            }
            // ---- broadcast receivers (SyncInSerial, simulation.cu:357-407)
            const int chan = s->chan;
            if (chan > 0) {
                const int sender = s->sender;
                uint32_t rm[K];
                bool any = false;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    rm[k] = 0;
                    const uint32_t c = c0 + k;
                    if (c < C && static_cast<int>(c) != sender && n.loc[loc[k]].n_recv) {
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
                            slots[k] = write_slots(slots[k], rm[k]);
                            if (VERIFY) mix(s->digest, c | 0x80000000u);
                            loc[k] = base + take<VERIFY>(n, s, p, run, step, c, loc[k] - base, rm[k], slots[k], 1);
                        }
                    }
                    __syncwarp(gmask);
                    pending &= pending - 1;
                }
                if (gl == 0) {
                    s->chan = 0;
                    s->sender = -1;
                }
                __syncwarp(gmask);
            }

            // ---- distinct rate programs, once per step per run
            if (rate_table) {
                for (uint32_t j = gl; j < n.n_rate_prog; j += G)
                    s->vars[V + j] = inv_rate(eval(n, s->vars, n.rate_prog[j]));
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
                        if (k % 4 == 0) blk = delay_block(p.seed, run, step, c >> 2);
                        x = word_of(blk, static_cast<uint32_t>(k & 3));
                    } else {
                        x = delay_word(p.seed, run, step, c);
                    }
                    const float d = comp_delay(n, s, loc[k], x);
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
                mix(s->digest, step);
                mix(s->digest, win);
                mix(s->digest, f_bits(dmin));
            }
            if (static_cast<double>(dmin) < kDblMax) {
                // clocks advance (simulation.cu:632-651)
                for (uint32_t v = gl; v < V; v += G)
                    if (n.var[v].kind)
                        s->vars[v] = d2f(d_add(static_cast<double>(s->vars[v]), static_cast<double>(dmin)));
                __syncwarp(gmask);
                if (gl == owner) {
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        if (c0 + k != win) continue;
                        const uint32_t base = n.comp[win].loc_begin;
                        loc[k] = base + win_step<VERIFY>(n, s, p, run, step, win, loc[k] - base, &slots[k]);
                    }
                }
                __syncwarp(gmask);
            }
            time = d2f(d_add(static_cast<double>(time), static_cast<double>(dmin)));  // simulation.cu:876-882
            ++step;
        }

        // per-run outputs (simulation.cu:887-893)
        if (gl == 0) {
            const double val = p.is_max ? s->qmax : s->qmin;
            uint32_t f = flag;
            if (!p.loc_mode) f = p.is_max ? (val > p.threshold) : (val < p.threshold);
            if (p.flags) p.flags[ridx] = static_cast<uint8_t>(f);
            if (p.values) p.values[ridx] = val;
            if (p.steps) p.steps[ridx] = step;
            if (VERIFY && p.digests) p.digests[ridx] = s->digest;
            acc_hits += f;
            acc_steps += step;
            acc_capped += capped;
        }
        if (VERIFY && p.final_state) {
            uint32_t *w = p.final_state + ridx * (C + V);
#pragma unroll
            for (int k = 0; k < K; ++k)
                if (c0 + k < C) w[c0 + k] = loc[k] - n.comp[c0 + k].loc_begin;
            for (uint32_t v = gl; v < V; v += G) w[C + v] = f_bits(s->vars[v]);
        }
        __syncwarp(gmask);
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
