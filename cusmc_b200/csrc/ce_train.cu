// Cross-entropy training of the importance-sampling proposal through the C
// ABI, for hosts without Python (the CLI's --csmc-is, C/C++ programs):
// csmc_is_train runs the whole multi-level CE loop on the GPU — runs under
// the current proposal (csmc_is_run), elite selection (csmc_ce_select),
// replay of the elite runs into training rows (csmc_is_trace), the row
// merge (csmc_mlp_rows_merge), Adam ascent on the tensor-core gradient, all
// steps of a round on the device (csmc_mlp_adam) — and returns the trained
// FP32 master parameters and a per-round log.
//
// The elite selection and the Adam steps are library code shared with the
// Python training loop (cusmc_b200/proposal.py calls csmc_ce_select and
// csmc_mlp_adam), so both loops select the same runs and take the same
// steps; the loop itself and the BF16 packing of the runs' parameters are
// written independently on both sides, and a GPU test requires the two
// trainings to end with the same parameters bit for bit.
#include "../../include/csmc.h"
#include "capi_internal.h"
#include "include/csmc_mlp.h"
#include "include/csmc_numeric.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <numeric>
#include <string>
#include <vector>

namespace {

int fail(int code, const std::string &m) {
    csmc::set_last_error(m);
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(CSMC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr int kHid = CSMC_MLP_HID, kIn = CSMC_MLP_IN;
constexpr int kFloats = CSMC_MLP_GRAD_FLOATS;  // master vector: w1, b1, w2, b2, w3, b3
constexpr size_t kRowBytes = sizeof(csmc::MlpRow);
static_assert(kRowBytes == 40, "training row layout");

struct Selection {
    std::vector<uint64_t> elite;
    std::vector<float> weights;
    std::vector<uint64_t> offsets;
    uint64_t n_rows = 0;
    double level = 0.0;
    bool at_goal = false;
};

// The multi-level CE selection of csmc_ce_select (see include/csmc.h).
Selection select(const double *values, const double *logw, const uint32_t *steps, uint64_t n, double threshold,
                 bool is_max, double rho, uint64_t max_rows) {
    Selection s;
    std::vector<double> score(n);
    for (uint64_t i = 0; i < n; ++i) score[i] = is_max ? values[i] : -values[i];
    const double goal = is_max ? threshold : -threshold;
    std::vector<double> sorted(score);
    std::sort(sorted.begin(), sorted.end());
    // (1 - rho)-quantile, linear interpolation between order statistics
    const double h = static_cast<double>(n - 1) * (1.0 - rho);
    const uint64_t lo = static_cast<uint64_t>(std::floor(h));
    const uint64_t hi = std::min<uint64_t>(lo + 1, n - 1);
    const double t = h - static_cast<double>(lo);
    const double q = sorted[lo] + (sorted[hi] - sorted[lo]) * t;
    const double level = std::min(goal + 1e-9, q);
    std::vector<uint64_t> elite;
    for (uint64_t i = 0; i < n; ++i)
        if (level <= goal ? score[i] >= level : score[i] > goal) elite.push_back(i);
    if (elite.empty()) {  // the highest-scoring runs, ascending by score (stable)
        std::vector<uint64_t> idx(n);
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) { return score[a] < score[b]; });
        const uint64_t k = std::max<uint64_t>(1, static_cast<uint64_t>(rho * static_cast<double>(n)));
        elite.assign(idx.end() - static_cast<std::ptrdiff_t>(k), idx.end());
    }
    // likelihood-ratio weights, normalised (sequential sums)
    const size_t m = elite.size();
    double mx = logw[elite[0]];
    for (uint64_t e : elite) mx = std::max(mx, logw[e]);
    std::vector<double> w(m);
    double sum = 0.0;
    for (size_t j = 0; j < m; ++j) {
        w[j] = std::exp(logw[elite[j]] - mx);
        sum += w[j];
    }
    for (size_t j = 0; j < m; ++j) w[j] = w[j] / sum;
    // heaviest first while the rows (four per step) fit the cap
    std::vector<size_t> order(m);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return w[a] > w[b]; });
    std::vector<size_t> keep;
    uint64_t rows = 0;
    for (size_t j : order) {
        rows += 4ull * steps[elite[j]];
        if (rows > max_rows) break;
        keep.push_back(j);
    }
    if (keep.empty()) keep.push_back(order[0]);
    double ksum = 0.0;
    for (size_t j : keep) ksum += w[j];
    uint64_t off = 0;
    for (size_t j : keep) {
        s.elite.push_back(elite[j]);
        s.weights.push_back(static_cast<float>(w[j] / ksum));
        s.offsets.push_back(off);
        off += 4ull * steps[elite[j]];
    }
    s.n_rows = off;
    s.level = is_max ? level : -level;
    s.at_goal = level > goal;
    return s;
}

// FP32 master vector -> the BF16 parameter block (csmc::MlpParams).
void pack(const float *x, csmc::MlpParams &P) {
    std::memset(&P, 0, sizeof P);
    int o = 0;
    for (int j = 0; j < kHid; ++j)
        for (int i = 0; i < kIn; ++i) P.w1[j][i] = csmc::f_to_bf16(x[o++]);
    for (int j = 0; j < kHid; ++j) P.b1[j] = x[o++];
    for (int k = 0; k < kHid; ++k)
        for (int j = 0; j < kHid; ++j) P.w2[k][j] = csmc::f_to_bf16(x[o++]);
    for (int k = 0; k < kHid; ++k) P.b2[k] = x[o++];
    for (int k = 0; k < kHid; ++k) P.w3[k] = x[o++];
    P.b3 = x[o++];
}

// Adam's moments and step count across the rounds (the steps themselves run
// on the device: csmc_mlp_adam).
struct AdamState {
    std::vector<double> m, v;
    int32_t t = 0;
    AdamState() : m(kFloats, 0.0), v(kFloats, 0.0) {}
};

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    ~DevBuf() { cudaFree(p); }
    cudaError_t ensure(size_t b) {
        if (b <= bytes) return cudaSuccess;
        cudaFree(p);
        p = nullptr;
        bytes = 0;
        const cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    template <class T>
    T *as() const {
        return static_cast<T *>(p);
    }
};

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int train(csmc_net *net, const csmc_query *q, uint64_t seed, const csmc_ce_config &cfg, const float *init,
          float *trained, void *params_out, csmc_ce_round *log, int32_t log_cap, int32_t *rounds_done) {
    if (q->kind != CSMC_QUERY_VARIABLE)
        return fail(CSMC_ERR_ARG, "CE training needs a variable query (the tracked value ranks the runs)");
    if (cfg.rounds < 1 || cfg.adam_steps < 1 || cfg.runs_per_round < 1 || !(cfg.rho > 0.0 && cfg.rho < 1.0) ||
        cfg.max_rows < 1)
        return fail(CSMC_ERR_ARG, "CE configuration: rounds, adam_steps, runs_per_round and max_rows must be "
                                  "positive and rho in (0, 1)");
    const uint64_t n = cfg.runs_per_round;
    std::vector<float> x(init, init + kFloats);
    AdamState opt;
    DevBuf d_flags, d_logw, d_values, d_steps, d_rows, d_merged, d_elite, d_w, d_off;
    cudaError_t e = d_flags.ensure(n);
    if (e == cudaSuccess) e = d_logw.ensure(n * sizeof(double));
    if (e == cudaSuccess) e = d_values.ensure(n * sizeof(double));
    if (e == cudaSuccess) e = d_steps.ensure(n * sizeof(uint32_t));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(CE round buffers)");
    std::vector<double> h_values(n), h_logw(n);
    std::vector<uint32_t> h_steps(n);
    csmc::MlpParams P;
    int at_goal = 0, done = 0;
    for (int32_t k = 0; k < cfg.rounds; ++k) {
        const auto t0 = std::chrono::steady_clock::now();
        pack(x.data(), P);
        const uint64_t first = static_cast<uint64_t>(k + 1) * 10000000ull;  // fresh runs every round
        csmc_result res{};
        int rc = csmc_is_run(net, q, &P, seed, first, n, d_flags.as<uint8_t>(), d_logw.as<double>(),
                             d_values.as<double>(), d_steps.as<uint32_t>(), &res, nullptr);
        if (rc) return rc;
        e = cudaMemcpy(h_values.data(), d_values.p, n * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(h_logw.data(), d_logw.p, n * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(h_steps.data(), d_steps.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "copy of the round's runs");
        const Selection s = select(h_values.data(), h_logw.data(), h_steps.data(), n, q->threshold, q->is_max != 0,
                                   cfg.rho, cfg.max_rows);
        const size_t m = s.elite.size();
        e = d_rows.ensure(std::max<uint64_t>(1, s.n_rows) * kRowBytes);
        if (e == cudaSuccess) e = d_merged.ensure(std::max<uint64_t>(1, s.n_rows) * kRowBytes);
        if (e == cudaSuccess) e = d_elite.ensure(m * sizeof(uint64_t));
        if (e == cudaSuccess) e = d_w.ensure(m * sizeof(float));
        if (e == cudaSuccess) e = d_off.ensure(m * sizeof(uint64_t));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(training rows)");
        e = cudaMemcpy(d_elite.p, s.elite.data(), m * sizeof(uint64_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_w.p, s.weights.data(), m * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_off.p, s.offsets.data(), m * sizeof(uint64_t), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "upload of the elite runs");
        const double run_s = seconds_since(t0);
        const auto t1 = std::chrono::steady_clock::now();
        rc = csmc_is_trace(net, q, &P, seed, first, d_elite.as<uint64_t>(), d_w.as<float>(), d_off.as<uint64_t>(), m,
                           d_rows.p, d_rows.bytes / kRowBytes, nullptr);
        if (rc) return rc;
        // rows of equal features on consecutive steps summed (J unchanged)
        uint64_t m_rows = 0;
        rc = csmc_mlp_rows_merge(d_rows.p, d_off.as<uint64_t>(), m, s.n_rows, d_merged.p, &m_rows, nullptr);
        if (rc) return rc;
        const double trace_s = seconds_since(t1);
        const auto t2 = std::chrono::steady_clock::now();
        double J0 = 0.0, J = 0.0;
        rc = csmc_mlp_adam(d_merged.p, m_rows, cfg.adam_steps, cfg.lr, x.data(), opt.m.data(), opt.v.data(), &opt.t,
                           &J0, &J, nullptr);
        if (rc) return rc;
        const double adam_s = seconds_since(t2);
        if (log && k < log_cap) {
            csmc_ce_round &L = log[k];
            std::memset(&L, 0, sizeof L);
            L.round = k;
            L.elite = static_cast<int32_t>(m);
            L.rows = s.n_rows;
            L.level = s.level;
            L.j_start = J0;
            L.j_end = J;
            L.estimate = res.estimate;
            L.hits = res.hits;
            L.capped = res.capped;
            L.mean_steps = static_cast<double>(res.steps) / static_cast<double>(res.runs ? res.runs : 1);
            L.kernel_ms = res.kernel_ms;
            L.run_s = run_s;
            L.trace_s = trace_s;
            L.adam_s = adam_s;
            L.at_goal = s.at_goal ? 1 : 0;
        }
        done = k + 1;
        at_goal = s.at_goal ? at_goal + 1 : 0;
        if (cfg.settle && at_goal >= cfg.settle) break;
    }
    std::memcpy(trained, x.data(), kFloats * sizeof(float));
    if (params_out) {
        pack(x.data(), P);
        std::memcpy(params_out, &P, sizeof P);
    }
    if (rounds_done) *rounds_done = done;
    return CSMC_OK;
}

}  // namespace

extern "C" {

int csmc_ce_select(const double *values, const double *logw, const uint32_t *steps, uint64_t n, double threshold,
                   int32_t is_max, double rho, uint64_t max_rows, uint64_t *elite, float *weights,
                   uint64_t *row_offset, uint64_t *n_elite, uint64_t *n_rows, double *level, int32_t *at_goal) {
    if (!values || !logw || !steps || !elite || !weights || !row_offset || !n_elite || !n_rows || !level || !at_goal)
        return fail(CSMC_ERR_ARG, "null argument");
    if (n == 0 || !(rho > 0.0 && rho < 1.0) || max_rows == 0)
        return fail(CSMC_ERR_ARG, "csmc_ce_select: n and max_rows must be positive and rho in (0, 1)");
    try {
        const Selection s = select(values, logw, steps, n, threshold, is_max != 0, rho, max_rows);
        std::copy(s.elite.begin(), s.elite.end(), elite);
        std::copy(s.weights.begin(), s.weights.end(), weights);
        std::copy(s.offsets.begin(), s.offsets.end(), row_offset);
        *n_elite = s.elite.size();
        *n_rows = s.n_rows;
        *level = s.level;
        *at_goal = s.at_goal ? 1 : 0;
        return CSMC_OK;
    } catch (const std::exception &ex) {
        return fail(CSMC_ERR_ARG, ex.what());
    }
}

int csmc_mlp_pack(const float *master, void *params) {
    if (!master || !params) return fail(CSMC_ERR_ARG, "null argument");
    csmc::MlpParams P;
    pack(master, P);
    std::memcpy(params, &P, sizeof P);
    return CSMC_OK;
}

int csmc_mlp_init(uint64_t seed, float *master) {
    if (!master) return fail(CSMC_ERR_ARG, "null argument");
    // normal draws by the Box-Muller transform of Philox4x32-10 uniforms
    // (stream (seed, block i)): w1 ~ N(0, 2/10) on the 10 used inputs, w2 ~
    // N(0, 2/64), everything else 0 (theta = 0: the nominal model)
    uint64_t blk = 0;
    auto normal_pair = [&](double &z0, double &z1) {
        const csmc::u32x4 r = csmc::philox4x32_10(csmc::u32x4{static_cast<uint32_t>(blk), static_cast<uint32_t>(blk >> 32),
                                                              0x6d6c7069u, 0u},
                                                  static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
        ++blk;
        const double u1 = (static_cast<double>(r.x) + 1.0) / 4294967296.0;  // (0, 1]
        const double u2 = static_cast<double>(r.y) / 4294967296.0;
        const double rad = std::sqrt(-2.0 * std::log(u1));
        z0 = rad * std::cos(6.283185307179586 * u2);
        z1 = rad * std::sin(6.283185307179586 * u2);
    };
    std::memset(master, 0, kFloats * sizeof(float));
    std::vector<double> z;
    auto next = [&]() {
        if (z.empty()) {
            double a, b;
            normal_pair(a, b);
            z.push_back(b);
            return a;
        }
        const double v = z.back();
        z.pop_back();
        return v;
    };
    int o = 0;
    for (int j = 0; j < kHid; ++j)
        for (int i = 0; i < kIn; ++i, ++o) master[o] = i < CSMC_MLP_FEATURES ? static_cast<float>(next() * std::sqrt(0.2)) : 0.0f;
    o += kHid;  // b1
    for (int k = 0; k < kHid * kHid; ++k, ++o) master[o] = static_cast<float>(next() * std::sqrt(2.0 / kHid));
    return CSMC_OK;
}

int csmc_is_train(csmc_net *net, const csmc_query *q, uint64_t seed, const csmc_ce_config *cfg, const float *init,
                  float *trained, void *params_out, csmc_ce_round *log, int32_t log_cap, int32_t *rounds_done) {
    if (!net || !q || !cfg || !init || !trained) return fail(CSMC_ERR_ARG, "null argument");
    try {
        return train(net, q, seed, *cfg, init, trained, params_out, log, log_cap, rounds_done);
    } catch (const std::exception &ex) {
        return fail(CSMC_ERR_ARG, ex.what());
    }
}

}  // extern "C"

namespace {

// The smc() report (smc.cu:283-402) for an importance-sampling estimate of a
// variable probability query: the settings block, the CE rounds, the
// estimate with its 95% interval and the timing lines.
int smc_is(const char *model_path, int seed, int sims, const csmc_query &q, const csmc_ce_config &cfg,
           const char *json_path) {
    if (q.kind != CSMC_QUERY_VARIABLE || q.is_estimate)
        return fail(CSMC_ERR_ARG, "importance sampling estimates a variable probability query "
                                  "(VAR_ID >= 0, IS_ESTIMATE = 0)");
    if (sims <= 0) return fail(CSMC_ERR_ARG, "the number of simulations must be positive");
    void *blob = nullptr;
    size_t bytes = 0;
    int rc = csmc_model_compile(model_path, "", 0, &blob, &bytes);
    if (rc) return rc;
    uint32_t n_vars = 0, n_comps = 0, n_locs = 0;
    csmc_blob_info(blob, bytes, &n_vars, &n_comps, &n_locs);
    std::printf("Set number of variables to: %d\n", static_cast<int>(n_vars));
    std::fflush(stdout);
    std::cout << "=================\n\n";
    std::cout << "Running SMC with the following settings:" << std::endl;
    std::cout << "- Number of simulations: " << sims << std::endl;
    std::cout << "- Model: " << model_path << std::endl;
    std::cout << "- Random seed: " << seed << std::endl;
    std::cout << "- Time bound: " << q.horizon << std::endl;
    std::cout << "- Num components: " << n_comps << std::endl;
    std::cout << "- Logging type: variable query. Finding " << (q.is_max ? "max" : "min") << " of variable with ID "
              << q.var_id << std::endl;
    std::cout << "- Importance sampling: learned proposal, up to " << cfg.rounds << " CE rounds of "
              << cfg.runs_per_round << " runs" << std::endl;
    std::cout << "=================\n\n";
    csmc_net *net = nullptr;
    rc = csmc_net_upload(blob, bytes, &net);
    std::free(blob);
    if (rc) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<float> init(kFloats), trained(kFloats);
    csmc::MlpParams P;
    std::vector<csmc_ce_round> log(static_cast<size_t>(cfg.rounds));
    int32_t done = 0;
    const uint64_t seed64 = static_cast<uint64_t>(static_cast<int64_t>(seed));
    rc = csmc_mlp_init(seed64, init.data());
    if (!rc) rc = csmc_is_train(net, &q, seed64, &cfg, init.data(), trained.data(), &P, log.data(), cfg.rounds, &done);
    if (rc) {
        csmc_net_free(net);
        return rc;
    }
    for (int32_t k = 0; k < done; ++k)
        std::cout << "CE round " << k << ": level " << log[k].level << ", elite runs " << log[k].elite
                  << ", training rows " << log[k].rows << ", estimate " << log[k].estimate << std::endl;
    const double train_ms = seconds_since(t0) * 1000.0;
    // the estimate: sims runs under the trained proposal, beyond the
    // training runs of the stream
    double s1 = 0.0, s2 = 0.0;
    uint64_t hits = 0;
    const uint64_t first = static_cast<uint64_t>(cfg.rounds + 2) * 10000000ull;
    for (uint64_t d = 0; d < static_cast<uint64_t>(sims);) {
        const uint64_t m = std::min<uint64_t>(static_cast<uint64_t>(sims) - d, 1u << 21);
        csmc_result r{};
        rc = csmc_is_run(net, &q, &P, seed64, first + d, m, nullptr, nullptr, nullptr, nullptr, &r, nullptr);
        if (rc) {
            csmc_net_free(net);
            return rc;
        }
        s1 += r.sum;
        s2 += r.sum_sq;
        hits += r.hits;
        d += m;
    }
    csmc_net_free(net);
    const auto dur = std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0);
    const double ms = dur.count() / 1000000.0;
    const double n = static_cast<double>(sims), p = s1 / n;
    const double half = 1.96 * std::sqrt(std::max(0.0, s2 / n - p * p) / n);
    std::cout << "Time taken: " << ms << " ms on file " << model_path << std::endl;
    std::cout << "Time taken: " << dur.count() << " on file " << model_path << std::endl;
    std::cout << "Time taken: " << dur.count() << " ns (" << ms << " ms)" << std::endl;
    std::cout << "Result: " << p << std::endl;
    std::cout << "95% confidence interval: [" << p - half << ", " << p + half << "] (relative half-width "
              << (p > 0 ? half / p : 0.0) << ")" << std::endl;
    if (json_path && *json_path) {
        std::ofstream o(json_path);
        if (!o) return fail(CSMC_ERR_ARG, std::string("cannot write ") + json_path);
        o << std::setprecision(17);
        o << "{\"model\": \"" << model_path << "\", \"seed\": " << seed << ", \"simulations\": " << sims
          << ", \"method\": \"importance sampling (learned proposal)\", \"query\": {\"var_id\": " << q.var_id
          << ", \"is_max\": " << q.is_max << ", \"threshold\": " << q.threshold << ", \"time_bound\": " << q.horizon
          << "}, \"result\": " << p << ", \"ci95\": [" << p - half << ", " << p + half << "], \"runs_at_goal\": "
          << hits << ", \"ce_rounds\": " << done << ", \"train_ms\": " << train_ms << ", \"ms\": " << ms
          << "}\n";
    }
    return CSMC_OK;
}

}  // namespace

extern "C" int csmc_smc_is(const char *model_path, int seed, int sims, const csmc_query *q,
                           const csmc_ce_config *cfg, const char *json_path) {
    if (!model_path || !q || !cfg) return fail(CSMC_ERR_ARG, "null argument");
    try {
        return smc_is(model_path, seed, sims, *q, *cfg, json_path);
    } catch (const std::exception &ex) {
        return fail(CSMC_ERR_ARG, ex.what());
    }
}
