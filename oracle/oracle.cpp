/*
 * CPU oracle — TEST INFRASTRUCTURE ONLY.  A single-threaded restatement of
 * the reference cuSMC simulation semantics over the packed network, used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker.  Nothing in the product (cusmc_b200, the CLI, libcsmc.so) links,
 * loads or calls it.
 *
 * Parity status: the front end that produces the packed network is pinned
 * byte-for-byte against the reference's own parser and passes (oracle/ref/
 * refdump.cpp, tests/golden/frontend).  The simulation semantics below
 * restate the reference kernel; they are pinned statistically against the
 * reference binary run on the GPU (tests/golden/ref_estimates.json) and by
 * closed forms.  The reference draws from curand states shared across blocks
 * (simulation/simulation.cu:756-760, smc.cu:228), so its runs have no
 * reproducible traces to compare bit for bit; traces are compared bit for bit
 * between this oracle and the CUDA kernels, which share only the numeric
 * spec of cusmc_b200/csrc/include/csmc_numeric.h.
 *
 * Step semantics followed (simulation/simulation.cu):
 *   loop / goal exit / time advance ............ 835-885
 *   broadcast receivers (serial, in order) ...... 357-407
 *   delay per component ......................... 409-541
 *   race: tree argmin, clock advance, winner .... 544-671
 *   edge enabling / guards ...................... 184-305
 *   edge choice, updates, destination, goal ..... 9-181
 *   per-run output ............................... 887-893
 * Expression evaluation: simulation/expressions.cu:88-229.
 */
#include "../include/csmc.h"
#include "../cusmc_b200/csrc/include/csmc_net.h"
#include "../cusmc_b200/csrc/include/csmc_numeric.h"
#include "../cusmc_b200/csrc/include/csmc_mlp.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

using namespace csmc;

namespace {

thread_local std::string g_err;

constexpr double kEps = 0.00001;
constexpr double kDblMax = 1.7976931348623158e+308;
constexpr double kDblMin = 2.2250738585072014e-308;

struct Net {
    const csmc_net_header *h;
    const csmc_comp *comp;
    const csmc_loc *loc;
    const csmc_edge *edge;
    const csmc_guard *guard;
    const csmc_update *upd;
    const csmc_var *var;
    const double *konst;
    const uint64_t *code;
};

Net view(const void *blob, size_t bytes) {
    if (!blob || bytes < sizeof(csmc_net_header)) throw std::runtime_error("blob too small");
    const uint8_t *b = static_cast<const uint8_t *>(blob);
    Net n;
    n.h = reinterpret_cast<const csmc_net_header *>(b);
    if (n.h->magic != CSMC_NET_MAGIC || n.h->total_bytes > bytes) throw std::runtime_error("not a network blob");
    n.comp = reinterpret_cast<const csmc_comp *>(b + n.h->off_comp);
    n.loc = reinterpret_cast<const csmc_loc *>(b + n.h->off_loc);
    n.edge = reinterpret_cast<const csmc_edge *>(b + n.h->off_edge);
    n.guard = reinterpret_cast<const csmc_guard *>(b + n.h->off_guard);
    n.upd = reinterpret_cast<const csmc_update *>(b + n.h->off_update);
    n.var = reinterpret_cast<const csmc_var *>(b + n.h->off_var);
    n.konst = reinterpret_cast<const double *>(b + n.h->off_const);
    n.code = reinterpret_cast<const uint64_t *>(b + n.h->off_code);
    return n;
}

struct Digest {
    uint64_t h = 0xcbf29ce484222325ull;
    void mix(uint32_t w) { h = (h ^ w) * 0x100000001b3ull; }
};

class Run {
  public:
    Run(const Net &n, const csmc_query &q, uint64_t seed, uint64_t run) : n_(n), q_(q), seed_(seed), run_(run) {}

    // expressions.cu:175-197 (PN, stack never popped by operators) and
    // expressions.cu:199-307 (tree evaluator)
    double eval(uint32_t h) const {
        const uint32_t tag = CSMC_H_TAG(h), p = CSMC_H_PAYLOAD(h);
        if (tag == CSMC_H_LIT) return n_.konst[p];
        if (tag == CSMC_H_VAR) return static_cast<double>(vars_[p]);
        double st[CSMC_MAX_STACK + 2];
        int top = 0;
        for (uint32_t ip = p;; ++ip) {
            const uint64_t ins = n_.code[ip];
            const uint32_t op = CSMC_INS_OP(ins), a = CSMC_INS_A(ins);
            double v1 = top >= 2 ? st[top - 2] : 0.0, v2 = top >= 1 ? st[top - 1] : 0.0;
            double r;
            switch (op) {
            case CSMC_OP_END: return top > 0 ? st[top - 1] : 0.0;
            case CSMC_OP_HDR: continue;
            case CSMC_OP_PUSH_C: r = n_.konst[a]; break;
            case CSMC_OP_PUSH_V: r = static_cast<double>(vars_[a]); break;
            case CSMC_OP_ADD: r = v1 + v2; break;
            case CSMC_OP_SUB: r = v1 - v2; break;
            case CSMC_OP_MUL: r = v1 * v2; break;
            case CSMC_OP_DIV: r = v1 / v2; break;
            case CSMC_OP_POW: r = pow_model(v1, v2); break;
            case CSMC_OP_NEG: r = -v2; break;
            case CSMC_OP_SQRT: r = std::sqrt(v2); break;
            case CSMC_OP_MOD: {
                const int x = d2i_sat(v1), y = d2i_sat(v2 + kEps);
                r = (y == 0 || (x == (-2147483647 - 1) && y == -1)) ? 0.0 : static_cast<double>(x % y);
                break;
            }
            case CSMC_OP_AND: r = (std::fabs(v1) > kEps && std::fabs(v2) > kEps) ? 1.0 : 0.0; break;
            case CSMC_OP_OR: r = (std::fabs(v1) > kEps || std::fabs(v2) > kEps) ? 1.0 : 0.0; break;
            case CSMC_OP_LE: r = v1 <= v2 ? 1.0 : 0.0; break;
            case CSMC_OP_GE: r = v1 >= v2 ? 1.0 : 0.0; break;
            case CSMC_OP_LT: r = v1 < v2 ? 1.0 : 0.0; break;
            case CSMC_OP_GT: r = v1 > v2 ? 1.0 : 0.0; break;
            case CSMC_OP_EQ: r = std::fabs(v1 - v2) <= kEps ? 1.0 : 0.0; break;
            case CSMC_OP_NE: r = std::fabs(v1 - v2) > kEps ? 1.0 : 0.0; break;
            case CSMC_OP_NOT: r = std::fabs(v2) < kEps ? 1.0 : 0.0; break;
            case CSMC_OP_RANDOM: r = 1.0; break;
            case CSMC_OP_DUP: r = v2; break;
            case CSMC_OP_ZERO: r = 0.0; break;
            case CSMC_OP_SKIP: {
                --top;
                if (std::fabs(st[top]) > kEps) ip += a;
                continue;
            }
            case CSMC_OP_TADD: case CSMC_OP_TSUB: case CSMC_OP_TMUL: case CSMC_OP_TDIV: {
                const double R = st[--top], L = st[--top];
                if (op == CSMC_OP_TADD) r = L + R;
                else if (op == CSMC_OP_TSUB) r = L - R;
                else if (op == CSMC_OP_TMUL) r = L * R;
                else if (R == 0.0) r = 0.0;
                else {
                    r = L / R;
                    if (r == 0.0) r = kDblMin;
                }
                break;
            }
            default: throw std::runtime_error("bad opcode");
            }
            st[top++] = r;
        }
    }

    // simulation.cu:184-266
    bool guards_ok(const csmc_edge &e) const {
        const uint32_t gb = CSMC_EDGE_GUARD_BEGIN(e), ng = CSMC_EDGE_N_GUARDS(e);
        for (uint32_t i = 0; i < ng; ++i) {
            const csmc_guard &g = n_.guard[gb + i];
            const double v = static_cast<double>(vars_[g.var]);
            const double b = eval(g.rhs);
            bool ok;
            switch (g.op) {
            case CSMC_G_LT: ok = v < b; break;
            case CSMC_G_LE: ok = v <= b; break;
            case CSMC_G_GT: ok = v > b; break;
            case CSMC_G_GE: ok = v >= b; break;
            case CSMC_G_EQ: ok = std::fabs(v - b) <= kEps; break;
            default: ok = false; break;
            }
            if (!ok) return false;
        }
        return true;
    }

    // simulation.cu:409-541
    float delay(uint32_t c) const {
        const csmc_loc &L = n_.loc[n_.comp[c].loc_begin + loc_[c]];
        if (L.type > 1) return 0.0f;
        double max_delay = kDblMax;
        bool bounded = false;
        for (uint32_t i = 0; i < L.n_inv; ++i) {
            const csmc_guard &g = n_.guard[L.inv_begin + i];
            const double cur = static_cast<double>(vars_[g.var]);
            const double bound = eval(g.rhs);
            double ttb = bound - cur;
            if (g.op == CSMC_G_LT) ttb -= 1e-6;
            if (ttb >= 0) {
                max_delay = std::fmin(max_delay, ttb);
                bounded = true;
            }
        }
        const uint32_t x = delay_word(seed_, run_, step_, c);
        if (bounded) return uniform_delay(x, max_delay);
        return exp_delay(x, inv_rate(eval(L.rate)));
    }

    // The delay under the importance-sampling proposal: exponential delays
    // of finite positive 1/rate are drawn with 1/rate multiplied by the
    // component's class factor e^(-theta).
    float delay_is(uint32_t c, const float *mfac, bool &tilted, float &inv, float &invp) const {
        tilted = false;
        inv = invp = 0.0f;
        const csmc_loc &L = n_.loc[n_.comp[c].loc_begin + loc_[c]];
        if (L.type > 1) return 0.0f;
        double max_delay = kDblMax;
        bool bounded = false;
        for (uint32_t i = 0; i < L.n_inv; ++i) {
            const csmc_guard &g = n_.guard[L.inv_begin + i];
            const double cur = static_cast<double>(vars_[g.var]);
            const double bound = eval(g.rhs);
            double ttb = bound - cur;
            if (g.op == CSMC_G_LT) ttb -= 1e-6;
            if (ttb >= 0) {
                max_delay = std::fmin(max_delay, ttb);
                bounded = true;
            }
        }
        const uint32_t x = delay_word(seed_, run_, step_, c);
        if (bounded) return uniform_delay(x, max_delay);
        inv = inv_rate(eval(L.rate));
        invp = inv;
        if (tiltable(inv)) {
            invp = f_mul(inv, mfac[loc_[c] & 3u]);
            tilted = true;
        }
        return exp_delay(x, invp);
    }

    // simulation.cu:9-24 and 27-181.  en: enabled edge indices (ascending).
    void take(uint32_t c, const std::vector<uint32_t> &en, uint32_t choice_which) {
        const uint32_t n = static_cast<uint32_t>(en.size());
        if (n == 0) return;
        const csmc_loc &L = n_.loc[n_.comp[c].loc_begin + loc_[c]];
        uint32_t sel = en[0];
        if (n > 1) {
            double sum = 0;
            for (uint32_t i = 0; i < L.n_edges; ++i)
                if ((mask_[c] >> i) & 1u) sum += eval(n_.edge[L.edge_begin + i].weight);
            const int W = d2i_sat(sum);
            const float u = uniform01(choice_word(seed_, run_, step_, c, choice_which));
            const int rnd = f2i_sat(f_mul(static_cast<float>(W), u));
            uint32_t temp = static_cast<uint32_t>(W);
            for (int i = static_cast<int>(n) - 1; i >= 0; --i) {
                const int w = d2i_sat(eval(n_.edge[L.edge_begin + i].weight));
                if (static_cast<int>(temp - static_cast<uint32_t>(w)) <= rnd) {
                    sel = en[i];
                    break;
                }
                temp -= static_cast<uint32_t>(w);
            }
        }
        if (digest_) {
            dg_.mix(sel);
        }
        const csmc_edge &e = n_.edge[L.edge_begin + sel];
        if (e.channel > 0) {
            chan_ = e.channel;
            sender_ = static_cast<int>(c);
        }
        const uint32_t ub = CSMC_EDGE_UPD_BEGIN(e), nu = CSMC_EDGE_N_UPD(e);
        for (uint32_t i = 0; i < nu; ++i) {
            const csmc_update &u = n_.upd[ub + i];
            const double nv = eval(u.expr);
            if (static_cast<int32_t>(u.var) == q_.var_id) {
                if (nv > qmax_) qmax_ = nv;
                if (nv < qmin_) qmin_ = nv;
            }
            vars_[u.var] = d2f(nv);
            if (digest_) {
                dg_.mix(u.var);
                dg_.mix(f_bits(vars_[u.var]));
            }
        }
        if (e.dst_local < 0) return;
        loc_[c] = static_cast<uint16_t>(e.dst_local);
        if (n_.loc[n_.comp[c].loc_begin + loc_[c]].type == CSMC_GOAL) goal_ = true;
    }

    // enabled-edge slot state: bit i <=> slot i holds edge index i
    void write_slots(uint32_t c, const std::vector<uint32_t> &en) {
        uint32_t m = mask_[c];
        for (uint32_t i = 0; i < en.size() && i < 32; ++i) {
            if (en[i] == i) m |= 1u << i;
            else m &= ~(1u << i);
        }
        mask_[c] = m;
    }

    void simulate(bool digest) {
        digest_ = digest;
        const uint32_t C = n_.h->n_comps, V = n_.h->n_vars;
        vars_.resize(V);
        for (uint32_t v = 0; v < V; ++v) vars_[v] = n_.var[v].init;
        loc_.resize(C);
        mask_.assign(C, 0u);
        for (uint32_t c = 0; c < C; ++c) loc_[c] = n_.comp[c].init_local;
        qmin_ = qmax_ = 0.0;
        if (q_.var_id >= 0 && static_cast<uint32_t>(q_.var_id) < V && n_.var[q_.var_id].kind == 0)
            qmin_ = qmax_ = static_cast<double>(n_.var[q_.var_id].init);
        const float T = static_cast<float>(q_.horizon);
        const uint64_t cap = q_.max_steps ? q_.max_steps : 10000000ull;
        const bool loc_mode = q_.kind == CSMC_QUERY_LOCATION;
        const uint32_t bits = ceil_log2(C);
        std::vector<float> d(C), inv(C), invp(C);
        std::vector<uint8_t> tilted(C);
        std::vector<uint32_t> keys(C), idx(C);
        std::vector<std::vector<uint32_t>> recv(C);
        std::vector<uint32_t> en;
        float time = 0.0f;
        while (time < T) {
            if (goal_ && loc_mode) {
                flag_ = 1;
                break;
            }
            if (step_ >= cap) {
                capped_ = true;
                break;
            }
            // broadcast receivers: enabled sets first, then serial transitions
            if (chan_ > 0) {
                for (uint32_t c = 0; c < C; ++c) {
                    recv[c].clear();
                    if (static_cast<int>(c) == sender_) continue;
                    const csmc_loc &L = n_.loc[n_.comp[c].loc_begin + loc_[c]];
                    for (uint32_t i = 0; i < L.n_edges; ++i) {
                        const csmc_edge &e = n_.edge[L.edge_begin + i];
                        if (e.channel == -chan_ && guards_ok(e)) recv[c].push_back(i);
                    }
                }
                for (uint32_t c = 0; c < C; ++c) {
                    if (recv[c].empty()) continue;
                    write_slots(c, recv[c]);
                    if (digest_) dg_.mix(c | 0x80000000u);
                    take(c, recv[c], 1);
                }
                chan_ = 0;
                sender_ = -1;
            }
            float mfac[CSMC_MLP_CLASSES] = {1.0f, 1.0f, 1.0f, 1.0f};
            float feat[CSMC_MLP_CLASSES][CSMC_MLP_IN];
            if (mlp_) {  // the proposal's class factors for this step
                float v4[4] = {0, 0, 0, 0};
                for (int i = 0; i < 4; ++i)
                    if (feat_.var[i] >= 0) v4[i] = vars_[feat_.var[i]];
                const float clk = feat_.clock_var >= 0 ? vars_[feat_.clock_var] : 0.0f;
                for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) {
                    mlp_features(l, feat_, v4, clk, time, T, feat[l]);
                    mfac[l] = tilt_factor(mlp_theta(*mlp_, feat[l]));
                }
            }
            for (uint32_t c = 0; c < C; ++c) {
                if (mlp_) {
                    bool t = false;
                    d[c] = delay_is(c, mfac, t, inv[c], invp[c]);
                    tilted[c] = t;
                } else {
                    d[c] = delay(c);
                }
                keys[c] = delay_key(d[c]);
                idx[c] = c;
            }
            // the reference's tree reduction (simulation.cu:576-628)
            uint32_t P = 1u << bits;
            for (uint32_t stride = P / 2; stride > 0; stride >>= 1)
                for (uint32_t t = 0; t < stride; ++t) {
                    const uint32_t j = t + stride;
                    if (j < C && keys[j] < keys[t]) {
                        keys[t] = keys[j];
                        idx[t] = idx[j];
                    }
                }
            const uint32_t win = idx[0];
            const float dmin = d[win];
            const bool finite = static_cast<double>(dmin) < kDblMax;
            // sums over components in warp order (csmc_mlp.h: warp_lane_of,
            // warp_tree_d), the order of the GPU kernel's one-warp-per-run step
            if (mlp_ && finite) {
                double part[CSMC_WARP] = {};
                for (uint32_t c = 0; c < C; ++c)
                    if (tilted[c]) part[warp_lane_of(c)] = d_add(part[warp_lane_of(c)], rate_change(inv[c], invp[c]));
                const double sum = warp_tree_d(part);
                logw_ = d_add(logw_, step_log_ratio(sum, dmin, tilted[win] != 0, inv[win], invp[win]));
            }
            if (mlp_ && rows_) {  // four rows per step, zero-weighted where nothing is tilted
                for (uint32_t l = 0; l < CSMC_MLP_CLASSES; ++l) {
                    double part[CSMC_WARP] = {};
                    uint32_t count = 0;
                    for (uint32_t c = 0; c < C; ++c)
                        if (tilted[c] && (loc_[c] & 3u) == l) {
                            part[warp_lane_of(c)] =
                                d_add(part[warp_lane_of(c)], d_div(1.0, static_cast<double>(inv[c])));
                            ++count;
                        }
                    const double inv_sum = warp_tree_d(part);
                    const bool has = finite && count > 0;
                    MlpRow r;
                    for (int i = 0; i < CSMC_MLP_IN; ++i) r.x[i] = f_to_bf16(feat[l][i]);
                    r.a = has ? row_a(inv_sum, dmin, row_w_) : 0.0f;
                    r.b = (has && tilted[win] && (loc_[win] & 3u) == l) ? row_w_ : 0.0f;
                    rows_->push_back(r);
                }
            }
            if (digest_) {
                dg_.mix(step_);
                dg_.mix(win);
                dg_.mix(f_bits(dmin));
            }
            if (static_cast<double>(dmin) < kDblMax) {
                for (uint32_t v = 0; v < V; ++v)
                    if (n_.var[v].kind) vars_[v] = d2f(static_cast<double>(vars_[v]) + static_cast<double>(dmin));
                const csmc_loc &L = n_.loc[n_.comp[win].loc_begin + loc_[win]];
                en.clear();
                for (uint32_t i = 0; i < L.n_edges; ++i) {
                    const csmc_edge &e = n_.edge[L.edge_begin + i];
                    if (e.channel >= 0 && guards_ok(e)) en.push_back(i);
                }
                write_slots(win, en);
                if (en.empty() && digest_) dg_.mix(0xffffffffu);
                take(win, en, 0);
            }
            time = d2f(static_cast<double>(time) + static_cast<double>(dmin));
            ++step_;
        }
        time_ = time;
    }

    const MlpParams *mlp_ = nullptr;   // importance sampling: the proposal network
    MlpFeatures feat_{};                // importance sampling: where its features come from
    double logw_ = 0.0;                 // log-likelihood ratio of the path
    std::vector<MlpRow> *rows_ = nullptr;  // replay: training rows
    float row_w_ = 0.0f;                // replay: the run's CE weight
    uint8_t flag_ = 0;
    bool capped_ = false;
    uint32_t step_ = 0;
    double qmin_ = 0, qmax_ = 0;
    float time_ = 0;
    std::vector<float> vars_;
    std::vector<uint16_t> loc_;
    uint64_t digest() const { return dg_.h; }

  private:
    const Net &n_;
    const csmc_query &q_;
    uint64_t seed_, run_;
    std::vector<uint32_t> mask_;
    bool goal_ = false;
    int chan_ = 0, sender_ = -1;
    bool digest_ = false;
    Digest dg_;
};

}  // namespace

extern "C" {

const char *oracle_last_error(void) { return g_err.c_str(); }

/* The numeric primitives on the host, over host arrays: the same function
 * codes and operand layouts as csmc_numeric_eval (include/csmc.h). */
int oracle_numeric_eval(int32_t fn, const void *a, const void *b, uint64_t n, void *out) {
    for (uint64_t i = 0; i < n; ++i) {
        switch (fn) {
        case CSMC_NUM_PHILOX: {
            const uint32_t *c = static_cast<const uint32_t *>(a) + 4 * i;
            const uint32_t *k = static_cast<const uint32_t *>(b) + 2 * i;
            const csmc::u32x4 r = csmc::philox4x32_10(csmc::u32x4{c[0], c[1], c[2], c[3]}, k[0], k[1]);
            uint32_t *o = static_cast<uint32_t *>(out) + 4 * i;
            o[0] = r.x;
            o[1] = r.y;
            o[2] = r.z;
            o[3] = r.w;
            break;
        }
        case CSMC_NUM_PHILOX_STEP: {
            const uint32_t *c = static_cast<const uint32_t *>(a) + 4 * i;
            const uint32_t *k = static_cast<const uint32_t *>(b) + 2 * i;
            const csmc::PhiloxKeys K = csmc::philox_keys(static_cast<uint64_t>(k[0]) | (static_cast<uint64_t>(k[1]) << 32));
            const csmc::PhiloxStep S = csmc::philox_step(K, c[0], static_cast<uint64_t>(c[2]) | (static_cast<uint64_t>(c[3]) << 32));
            const csmc::u32x4 r = csmc::philox_block(K, S, c[1]);
            uint32_t *o = static_cast<uint32_t *>(out) + 4 * i;
            o[0] = r.x;
            o[1] = r.y;
            o[2] = r.z;
            o[3] = r.w;
            break;
        }
        case CSMC_NUM_EXP_DELAY:
            static_cast<float *>(out)[i] =
                csmc::exp_delay(static_cast<const uint32_t *>(a)[i], static_cast<const float *>(b)[i]);
            break;
        case CSMC_NUM_LOG2_F32:
            static_cast<float *>(out)[i] = csmc::log2_pos(static_cast<const float *>(a)[i]);
            break;
        case CSMC_NUM_LOG2_F64:
            static_cast<double *>(out)[i] = csmc::log2_d(static_cast<const double *>(a)[i]);
            break;
        case CSMC_NUM_EXP2_F64:
            static_cast<double *>(out)[i] = csmc::exp2_d(static_cast<const double *>(a)[i]);
            break;
        case CSMC_NUM_POW_F64:
            static_cast<double *>(out)[i] =
                csmc::pow_model(static_cast<const double *>(a)[i], static_cast<const double *>(b)[i]);
            break;
        case CSMC_NUM_EXP2_F32:
            static_cast<float *>(out)[i] = csmc::exp2_f(static_cast<const float *>(a)[i]);
            break;
        case CSMC_NUM_GELU_F32:
            static_cast<float *>(out)[i] = csmc::gelu_f(static_cast<const float *>(a)[i]);
            break;
        case CSMC_NUM_GELU_GRAD_F32:
            static_cast<float *>(out)[i] = csmc::gelu_grad_f(static_cast<const float *>(a)[i]);
            break;
        default:
            g_err = "unknown numeric function";
            return -1;
        }
    }
    return 0;
}

/* Simulates runs with the reference semantics on `threads` host threads
 * (<= 0: all hardware threads).  Per-run outputs (host, may be NULL): flags,
 * values, steps, digests, final_state (n_comps + n_vars words per run).
 * wall_ms (may be NULL) receives the time spent in the run loop. */
int oracle_run(const void *blob, size_t bytes, const csmc_query *q, uint64_t seed, uint64_t first_run,
               uint64_t n_runs, int threads, uint8_t *flags, double *values, uint32_t *steps, uint64_t *digests,
               uint32_t *final_state, csmc_result *out, double *wall_ms) {
    try {
        if (!q) throw std::runtime_error("null query");
        const Net n = view(blob, bytes);
        const uint32_t C = n.h->n_comps, V = n.h->n_vars;
        if (q->kind == CSMC_QUERY_VARIABLE && (q->var_id < 0 || static_cast<uint32_t>(q->var_id) >= V))
            throw std::runtime_error("query variable id out of range");
        int nt = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
        if (nt < 1) nt = 1;
        if (static_cast<uint64_t>(nt) > n_runs) nt = static_cast<int>(std::max<uint64_t>(1, n_runs));
        std::vector<uint8_t> f(n_runs);
        std::vector<double> val(n_runs);
        std::vector<uint32_t> st(n_runs);
        std::vector<uint8_t> cap(n_runs);
        std::atomic<uint64_t> next{0};
        const bool want_digest = digests != nullptr;
        auto worker = [&]() {
            for (;;) {
                const uint64_t i = next.fetch_add(1);
                if (i >= n_runs) break;
                Run r(n, *q, seed, first_run + i);
                r.simulate(want_digest);
                const double v = q->is_max ? r.qmax_ : r.qmin_;
                uint8_t fl;
                if (q->kind == CSMC_QUERY_LOCATION) fl = r.flag_;
                else fl = q->is_max ? (v > q->threshold) : (v < q->threshold);
                f[i] = fl;
                val[i] = v;
                st[i] = r.step_;
                cap[i] = r.capped_ ? 1 : 0;
                if (digests) digests[i] = r.digest();
                if (final_state) {
                    uint32_t *w = final_state + i * (C + V);
                    for (uint32_t c = 0; c < C; ++c) w[c] = r.loc_[c];
                    for (uint32_t v2 = 0; v2 < V; ++v2) w[C + v2] = f_bits(r.vars_[v2]);
                }
            }
        };
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
        worker();
        for (auto &t : pool) t.join();
        const auto t1 = std::chrono::steady_clock::now();
        if (wall_ms) *wall_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        csmc_result res;
        std::memset(&res, 0, sizeof res);
        res.runs = n_runs;
        for (uint64_t i = 0; i < n_runs; ++i) {
            res.hits += f[i];
            res.steps += st[i];
            res.capped += cap[i];
            res.sum += val[i];
            res.sum_sq += val[i] * val[i];
        }
        if (n_runs) {
            if (q->kind == CSMC_QUERY_VARIABLE && q->is_estimate) res.estimate = res.sum / static_cast<double>(n_runs);
            else res.estimate = static_cast<double>(res.hits) / static_cast<double>(n_runs);
        }
        if (flags) std::memcpy(flags, f.data(), n_runs);
        if (values) std::memcpy(values, val.data(), n_runs * sizeof(double));
        if (steps) std::memcpy(steps, st.data(), n_runs * sizeof(uint32_t));
        if (out) *out = res;
        return CSMC_OK;
    } catch (const std::exception &e) {
        g_err = e.what();
        return CSMC_ERR_ARG;
    }
}

/* Full state after every step of one run: per step
 * [step, winner, delay bits, time bits, locations..., variable bits...]. */
int oracle_trace(const void *blob, size_t bytes, const csmc_query *q, uint64_t seed, uint64_t run,
                 uint32_t *rec, size_t cap_steps, size_t *n_steps) {
    try {
        const Net n = view(blob, bytes);
        csmc_query qq = *q;
        size_t k = 0;
        const uint32_t C = n.h->n_comps, V = n.h->n_vars;
        const size_t W = 4 + C + V;
        for (uint64_t s = 1;; ++s) {
            qq.max_steps = s;
            Run r(n, qq, seed, run);
            r.simulate(false);
            if (r.step_ < s || !r.capped_) {  // run ended before step s
                *n_steps = k;
                return CSMC_OK;
            }
            if (k < cap_steps) {
                uint32_t *w = rec + k * W;
                w[0] = static_cast<uint32_t>(s - 1);
                w[1] = 0;
                w[2] = 0;
                w[3] = f_bits(r.time_);
                for (uint32_t c = 0; c < C; ++c) w[4 + c] = r.loc_[c];
                for (uint32_t v = 0; v < V; ++v) w[4 + C + v] = f_bits(r.vars_[v]);
            }
            ++k;
            if (k >= cap_steps) {
                *n_steps = k;
                return CSMC_OK;
            }
        }
    } catch (const std::exception &e) {
        g_err = e.what();
        return CSMC_ERR_ARG;
    }
}

// The feature source of a run: features (may be NULL: the default of the network).
static MlpFeatures features_of(const Net &n, const void *features) {
    if (features) {
        MlpFeatures F;
        std::memcpy(&F, features, sizeof F);
        return F;
    }
    return mlp_default_features(n.h->n_vars, n.h->n_comps);
}

/* Importance sampling under the proposal network P (host MlpParams) with
 * the feature source features (csmc::MlpFeatures, may be NULL: the
 * default): per run (host, may be NULL): flags, log-likelihood ratios
 * (nominal over proposal), tracked values, steps.  Threads as oracle_run. */
int oracle_is_run(const void *blob, size_t bytes, const csmc_query *q, const void *params, const void *features,
                  uint64_t seed, uint64_t first_run, uint64_t n_runs, int threads, uint8_t *flags, double *logw,
                  double *values, uint32_t *steps, double *wall_ms) {
    try {
        if (!q || !params) throw std::runtime_error("null argument");
        const Net n = view(blob, bytes);
        const MlpParams *P = static_cast<const MlpParams *>(params);
        const MlpFeatures F = features_of(n, features);
        int nt = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
        if (nt < 1) nt = 1;
        if (static_cast<uint64_t>(nt) > n_runs) nt = static_cast<int>(std::max<uint64_t>(1, n_runs));
        std::atomic<uint64_t> next{0};
        auto worker = [&]() {
            for (;;) {
                const uint64_t i = next.fetch_add(1);
                if (i >= n_runs) break;
                Run r(n, *q, seed, first_run + i);
                r.mlp_ = P;
                r.feat_ = F;
                r.simulate(false);
                const double val = q->is_max ? r.qmax_ : r.qmin_;
                uint8_t f = r.flag_;
                if (q->kind == CSMC_QUERY_VARIABLE) f = q->is_max ? (val > q->threshold) : (val < q->threshold);
                if (flags) flags[i] = f;
                if (logw) logw[i] = r.logw_;
                if (values) values[i] = val;
                if (steps) steps[i] = r.step_;
            }
        };
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
        worker();
        for (auto &th : pool) th.join();
        if (wall_ms)
            *wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return CSMC_OK;
    } catch (const std::exception &e) {
        g_err = e.what();
        return CSMC_ERR_ARG;
    }
}

/* Replays runs first_run + runs[i] under P and appends their training rows
 * (weighted by weights[i]) in run-list order to rows (capacity cap rows);
 * *n_rows receives the number written (CSMC_ERR_LIMIT when cap is short). */
int oracle_is_trace(const void *blob, size_t bytes, const csmc_query *q, const void *params, const void *features,
                    uint64_t seed, uint64_t first_run, const uint64_t *runs, const float *weights, uint64_t n_list,
                    void *rows, uint64_t cap, uint64_t *n_rows) {
    try {
        const Net n = view(blob, bytes);
        const MlpParams *P = static_cast<const MlpParams *>(params);
        const MlpFeatures F = features_of(n, features);
        std::vector<MlpRow> out;
        for (uint64_t i = 0; i < n_list; ++i) {
            Run r(n, *q, seed, first_run + runs[i]);
            r.mlp_ = P;
            r.feat_ = F;
            r.rows_ = &out;
            r.row_w_ = weights[i];
            r.simulate(false);
        }
        *n_rows = out.size();
        if (out.size() > cap) {
            g_err = "row buffer too small";
            return CSMC_ERR_LIMIT;
        }
        std::memcpy(rows, out.data(), out.size() * sizeof(MlpRow));
        return CSMC_OK;
    } catch (const std::exception &e) {
        g_err = e.what();
        return CSMC_ERR_ARG;
    }
}

/* theta of one feature row (16 floats). */
float oracle_mlp_theta(const void *params, const float *x) {
    return mlp_theta(*static_cast<const MlpParams *>(params), x);
}

/* Gradient of J = sum over rows of (b theta - a e^theta) with respect to the
 * network's parameters, with the tensor-core kernels' roundings (first-layer
 * activations and the back-propagated pre-activation gradients in BF16),
 * accumulated in double.  grad (floats): w1[64][16], b1[64], w2[64][64],
 * b2[64], w3[64], b3.  objective receives J. */
int oracle_mlp_grad(const void *params, const void *rows_v, uint64_t n_rows, float *grad, double *objective) {
    const MlpParams &P = *static_cast<const MlpParams *>(params);
    const MlpRow *rows = static_cast<const MlpRow *>(rows_v);
    constexpr int H = CSMC_MLP_HID, I = CSMC_MLP_IN;
    std::vector<double> gw1(H * I, 0.0), gb1(H, 0.0), gw2(H * H, 0.0), gb2(H, 0.0), gw3(H, 0.0);
    double gb3 = 0.0, J = 0.0;
    float x[I], z1[H], h1[H], z2[H], h2[H], dz2b[H], dz1b[H];
    for (uint64_t r = 0; r < n_rows; ++r) {
        for (int i = 0; i < I; ++i) x[i] = bf16_to_f(rows[r].x[i]);
        for (int j = 0; j < H; ++j) {
            float z = P.b1[j];
            for (int i = 0; i < I; ++i) z = f_fma(x[i], bf16_to_f(P.w1[j][i]), z);
            z1[j] = z;
            h1[j] = bf16_round(gelu_f(z));
        }
        float th = P.b3;
        for (int k = 0; k < H; ++k) {
            float z = P.b2[k];
            for (int j = 0; j < H; ++j) z = f_fma(h1[j], bf16_to_f(P.w2[k][j]), z);
            z2[k] = z;
            h2[k] = gelu_f(z);
            th = f_fma(h2[k], P.w3[k], th);
        }
        const bool inside = th >= -CSMC_MLP_THETA_MAX && th <= CSMC_MLP_THETA_MAX;
        const float thc = inside ? th : (th < 0 ? -CSMC_MLP_THETA_MAX : CSMC_MLP_THETA_MAX);
        const float e = exp2_f(f_mul(thc, 1.44269502f));
        J += static_cast<double>(rows[r].b) * thc - static_cast<double>(rows[r].a) * e;
        const float g = inside ? f_add(rows[r].b, -f_mul(rows[r].a, e)) : 0.0f;
        if (g == 0.0f) continue;
        gb3 += g;
        for (int k = 0; k < H; ++k) {
            gw3[k] += static_cast<double>(g) * h2[k];
            dz2b[k] = bf16_round(f_mul(f_mul(g, P.w3[k]), gelu_grad_f(z2[k])));
            gb2[k] += dz2b[k];
            for (int j = 0; j < H; ++j) gw2[k * H + j] += static_cast<double>(dz2b[k]) * h1[j];
        }
        for (int j = 0; j < H; ++j) {
            double dh = 0.0;
            for (int k = 0; k < H; ++k) dh += static_cast<double>(dz2b[k]) * bf16_to_f(P.w2[k][j]);
            dz1b[j] = bf16_round(f_mul(static_cast<float>(dh), gelu_grad_f(z1[j])));
            gb1[j] += dz1b[j];
            for (int i = 0; i < I; ++i) gw1[j * I + i] += static_cast<double>(dz1b[j]) * x[i];
        }
    }
    float *o = grad;
    for (double v : gw1) *o++ = static_cast<float>(v);
    for (double v : gb1) *o++ = static_cast<float>(v);
    for (double v : gw2) *o++ = static_cast<float>(v);
    for (double v : gb2) *o++ = static_cast<float>(v);
    for (double v : gw3) *o++ = static_cast<float>(v);
    *o = static_cast<float>(gb3);
    if (objective) *objective = J;
    return CSMC_OK;
}

}  // extern "C"
