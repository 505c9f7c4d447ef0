// C ABI of importance sampling: runs under the proposal network, replay of
// listed runs into CE training rows, and the tensor-core gradient of the CE
// objective (mlp_train.cu).
#include "../../include/csmc.h"
#include "capi_internal.h"
#include "include/csmc_mlp.h"
#include "include/csmc_net.h"
#include "kernels/reduce.cuh"
#include "kernels/sim.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
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

#define CK(x, what)                                        \
    do {                                                   \
        cudaError_t e_ = (x);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

__global__ void reduce_weights(const double *w, uint64_t n, double *partials) {
    csmc::reduce_block(w, n, blockIdx.x, partials + 2 * blockIdx.x);
}

// Per-handle buffers of the importance-sampling path (lazily grown).
int ensure_is_buffers(csmc_net *n, uint64_t runs) {
    if (!n->d_mlp) CK(cudaMalloc(&n->d_mlp, sizeof(csmc::MlpParams)), "cudaMalloc(proposal network)");
    if (runs > n->is_cap) {
        cudaFree(n->d_wvals);
        cudaFree(n->d_is_flags);
        n->d_wvals = nullptr;
        n->d_is_flags = nullptr;
        n->is_cap = 0;
        CK(cudaMalloc(&n->d_wvals, runs * sizeof(double)), "cudaMalloc(weights)");
        CK(cudaMalloc(&n->d_is_flags, runs), "cudaMalloc(flags)");
        n->is_cap = runs;
    }
    return CSMC_OK;
}

struct Launch {
    int grid = 0, block = CSMC_IS_BLOCK;
    size_t smem = 0;
    uint32_t slab = 0;  // shared-memory bytes per warp (one run)
    bool slots = false, loc8 = false;
};

// One run per warp: the network and the proposal network once per CTA, then
// one slab per warp; CTAs of fewer warps when the slabs do not fit.
int plan_is(const csmc_net *n, bool trace, uint64_t n_runs, Launch &L) {
    const csmc_net_header &h = n->h;
    L.slots = h.max_edges_per_loc >= 2;
    L.loc8 = h.max_locs_per_comp <= 256;
    const size_t per = csmc::serial_state_bytes_per_thread(h.n_comps, h.n_vars, h.n_rate_prog, L.slots, L.loc8);
    L.slab = static_cast<uint32_t>(csmc::is_warp_slab_bytes(per, n->is_tc));
    const size_t base = n->bytes + csmc::is_mlp_smem_bytes();
    int max_smem = 0, sms = 0, ctas = 0;
    CK(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, n->device), "device attribute");
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n->device), "device attribute");
    int warps = CSMC_IS_BLOCK / 32;
    while (warps > 1 && base + static_cast<size_t>(warps) * L.slab > static_cast<size_t>(max_smem)) warps /= 2;
    L.block = 32 * warps;
    L.smem = base + static_cast<size_t>(warps) * L.slab;
    if (L.smem > static_cast<size_t>(max_smem))
        return fail(CSMC_ERR_LIMIT, "importance sampling needs the network, the proposal network and one run's "
                                    "state in shared memory (" + std::to_string(L.smem) + " bytes)");
    int rc = csmc::is_max_active_ctas(n->is_tc, trace, L.slots, L.loc8, L.block, L.smem, &ctas);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "occupancy query");
    if (ctas < 1) return fail(CSMC_ERR_LIMIT, "importance-sampling kernel cannot be resident");
    uint64_t grid = static_cast<uint64_t>(sms) * ctas;
    const uint64_t needed = (n_runs + warps - 1) / warps;
    if (grid > needed) grid = needed;
    L.grid = static_cast<int>(grid);
    return CSMC_OK;
}

// One thread per run (sim_is_coded.cuh) where the network has tilt groups,
// theta is evaluated on CUDA cores and the CTA's state fits; false: the
// one-warp-per-run kernel runs.
bool plan_is_coded(const csmc_net *n, uint64_t n_runs, Launch &L) {
    if (n->is_kernel == 3 || n->is_tc || n->is_groups < 0) return false;
    const csmc_net_header &h = n->h;
    L.slots = h.max_edges_per_loc >= 2;
    L.loc8 = true;
    int max_smem = 0, sms = 0, ctas = 0;
    if (cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, n->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n->device) != cudaSuccess)
        return false;
    // a small launch is bound by its single runs' steps, which one warp per
    // run takes faster.  The crossover, measured on the epidemic under a
    // trained proposal: with every location in a tilt group (no descriptor
    // path), one thread per run takes ~45 ms per launch up to a full GPU
    // and one warp per run ~6.1 us per run (5e3 runs: 44.5 against 33.4 ms;
    // 1e4 runs: 45.3 against 60.8 ms), so one thread per run from 48 runs
    // per SM; with the descriptor path, from 128 runs per SM (1e4 runs:
    // 134k runs/s against 165k; 2e4 runs: 242k against 179k)
    const uint64_t min_runs = (n->is_all_grouped ? 48ull : 128ull) * static_cast<uint64_t>(sms);
    if (n->is_kernel == 0 && n_runs < min_runs) return false;
    // threads per CTA: 384 (one CTA, twelve warps per SM) from 1.5 runs
    // per thread of such a grid, 128 (two CTAs per SM) when the runs fill
    // two of those per SM; a launch of fewer runs is bound by the steps of
    // single runs, and smaller CTAs (64, 32) spread its warps over more SMs.
    // Measured on the epidemic under a trained proposal: 1e6 runs 1.27M
    // runs/s with 384 threads against 1.04M with 128; 1e5 runs 886k
    // against 901k, and ten CE rounds of 1e5 runs 3.6 % faster in all
    const bool recv = (h.recv_chan_lo | h.recv_chan_hi) != 0;
    auto smem_of = [&](int block) {
        return n->bytes + csmc::is_coded_mlp_smem_bytes() + (block / 32) * csmc::is_coded_warp_smem_bytes() +
               csmc::is_coded_slab_bytes(h.n_comps, h.n_vars, h.n_rate_prog, L.slots, block,
                                         static_cast<uint32_t>(n->is_groups), recv);
    };
    auto resident = [&](int block) {  // CTAs per SM, 0 when it does not fit
        int c = 0;
        const size_t sm = smem_of(block);
        if (sm > static_cast<size_t>(max_smem)) return 0;
        if (csmc::is_coded_max_active_ctas(L.slots, n->is_all_grouped, block, sm, &c) != 0) {
            cudaGetLastError();
            return 0;
        }
        return c;
    };
    L.block = 0;
    if (n_runs >= 576ull * sms) {
        ctas = resident(384);
        if (ctas >= 1) L.block = 384;
    }
    if (L.block == 0 && n_runs >= 2ull * sms * 128) {
        ctas = resident(128);
        if (ctas >= 1) L.block = 128;
    }
    if (L.block == 0) {
        L.block = n_runs >= 2ull * sms * 64 ? 64 : 32;
        ctas = resident(L.block);
        if (ctas < 1) return false;
    }
    L.smem = smem_of(L.block);
    uint64_t grid = static_cast<uint64_t>(sms) * ctas;
    const uint64_t needed = (n_runs + L.block - 1) / L.block;
    if (grid > needed) grid = needed;
    L.grid = static_cast<int>(grid);
    L.slab = 0;
    return true;
}

// The theta cache of the thread-per-run kernel: 2^22 entries of 32 bytes,
// allocated on first use; a new generation (every entry free) whenever the
// parameter block differs from the one of the current generation.
constexpr uint32_t kThetaCacheEntries = 1u << 22;

int theta_cache_for(csmc_net *n, const void *params, cudaStream_t st) {
    const size_t bytes = static_cast<size_t>(kThetaCacheEntries) * CSMC_THETA_CACHE_WORDS * sizeof(uint32_t);
    if (!n->d_theta_cache) {
        CK(cudaMalloc(&n->d_theta_cache, bytes), "cudaMalloc(theta cache)");
        CK(cudaMemsetAsync(n->d_theta_cache, 0, bytes, st), "cudaMemsetAsync(theta cache)");
        n->theta_gen = 0;
    }
    if (n->theta_gen != 0 && std::memcmp(n->theta_params, params, CSMC_MLP_PARAM_BYTES) == 0) return CSMC_OK;
    if (n->theta_gen >= 0x7fffffffu) {  // generations run out: clear the states
        CK(cudaMemsetAsync(n->d_theta_cache, 0, bytes, st), "cudaMemsetAsync(theta cache)");
        n->theta_gen = 0;
    }
    ++n->theta_gen;
    std::memcpy(n->theta_params, params, CSMC_MLP_PARAM_BYTES);
    return CSMC_OK;
}

csmc::IsParams base_params(const csmc_net *n, const csmc_query *q, uint64_t seed, uint64_t first_run,
                           uint64_t n_runs) {
    csmc::IsParams ip{};
    csmc::SimParams &p = ip.s;
    p.net = csmc::layout_of(n->h);
    p.blob = n->d_blob;
    p.blob_bytes = n->bytes;
    p.loc_mode = q->kind == CSMC_QUERY_LOCATION;
    p.var_id = q->var_id;
    p.is_max = q->is_max;
    p.threshold = q->threshold;
    p.horizon = static_cast<float>(q->horizon);
    p.max_steps = q->max_steps ? q->max_steps : 10000000ull;
    p.seed = seed;
    p.first_run = first_run;
    p.n_runs = n_runs;
    p.scratch = n->d_scratch;
    p.keys = csmc::philox_keys(seed);
    ip.mlp = n->d_mlp;
    ip.feat = n->is_feat_set ? n->is_feat : csmc::mlp_default_features(n->h.n_vars, n->h.n_comps);
    ip.n_groups = n->is_groups > 0 ? static_cast<uint32_t>(n->is_groups) : 0u;
    ip.group_map = n->is_group_map;
    ip.group_l = n->is_group_l;
    for (int g = 0; g < CSMC_IS_GROUPS; ++g) ip.group_src[g] = n->is_group_src[g];
    return ip;
}

int check_query(const csmc_net *n, const csmc_query *q) {
    if (q->kind != CSMC_QUERY_LOCATION && q->kind != CSMC_QUERY_VARIABLE) return fail(CSMC_ERR_ARG, "bad query kind");
    if (q->kind == CSMC_QUERY_VARIABLE && (q->var_id < 0 || static_cast<uint32_t>(q->var_id) >= n->h.n_vars))
        return fail(CSMC_ERR_ARG, "query variable id out of range");
    return CSMC_OK;
}

}  // namespace

extern "C" {

int csmc_is_set_inference(csmc_net *n, int32_t tensor_cores) {
    if (!n) return fail(CSMC_ERR_ARG, "null argument");
    n->is_tc = tensor_cores != 0;
    return CSMC_OK;
}

int csmc_is_set_kernel(csmc_net *n, int32_t family) {
    if (!n) return fail(CSMC_ERR_ARG, "null argument");
    if (family != 0 && family != 3 && family != 5)
        return fail(CSMC_ERR_ARG, "importance-sampling kernel family must be 0, 3 or 5");
    n->is_kernel = family;
    return CSMC_OK;
}

int csmc_is_set_features(csmc_net *n, const int32_t *count_vars, const float *scales, int32_t clock_var) {
    if (!n) return fail(CSMC_ERR_ARG, "null argument");
    if (!count_vars && !scales && clock_var < 0) {
        n->is_feat_set = false;
        return CSMC_OK;
    }
    csmc::MlpFeatures F = csmc::mlp_default_features(n->h.n_vars, n->h.n_comps);
    for (int i = 0; i < 4; ++i) {
        if (count_vars) F.var[i] = count_vars[i] < 0 ? -1 : count_vars[i];
        if (scales) F.scale[i] = scales[i];
        if (F.var[i] >= 0 && static_cast<uint32_t>(F.var[i]) >= n->h.n_vars)
            return fail(CSMC_ERR_ARG, "feature variable id " + std::to_string(F.var[i]) + " out of range");
        if (!(F.scale[i] == F.scale[i]) || F.scale[i] > 3.0e38f || F.scale[i] < -3.0e38f)
            return fail(CSMC_ERR_ARG, "feature scales must be finite");
    }
    if (clock_var >= 0 && static_cast<uint32_t>(clock_var) >= n->h.n_vars)
        return fail(CSMC_ERR_ARG, "clock feature variable id out of range");
    F.clock_var = clock_var < 0 ? -1 : clock_var;
    n->is_feat = F;
    n->is_feat_set = true;
    return CSMC_OK;
}

int csmc_is_run(csmc_net *n, const csmc_query *q, const void *params, uint64_t seed, uint64_t first_run,
                uint64_t n_runs, uint8_t *flags, double *logw, double *values, uint32_t *steps, csmc_result *out,
                void *stream) {
    if (!n || !q || !params || !out) return fail(CSMC_ERR_ARG, "null argument");
    int rc = check_query(n, q);
    if (rc) return rc;
    if (first_run + n_runs < first_run || first_run + n_runs > (1ull << 62))
        return fail(CSMC_ERR_ARG, "run range out of bounds");
    std::memset(out, 0, sizeof *out);
    out->runs = n_runs;
    out->lanes_per_run = 32;
    out->comps_per_lane = static_cast<int32_t>((n->h.n_comps + 31) / 32);
    out->runs_per_cta = CSMC_IS_BLOCK / 32;
    out->family = 3;
    if (n_runs == 0) return CSMC_OK;
    CK(cudaSetDevice(n->device), "cudaSetDevice");
    rc = ensure_is_buffers(n, n_runs);
    if (rc) return rc;
    Launch L;
    const bool coded = plan_is_coded(n, n_runs, L);
    if (!coded) {
        rc = plan_is(n, false, n_runs, L);
        if (rc) return rc;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CK(cudaMemcpyAsync(n->d_mlp, params, sizeof(csmc::MlpParams), cudaMemcpyHostToDevice, st), "upload proposal");
    CK(cudaMemsetAsync(n->d_scratch, 0, CSMC_SCRATCH_WORDS * sizeof(unsigned long long), st), "cudaMemsetAsync");
    out->runs_per_cta = coded ? L.block : L.block / 32;
    if (coded) {
        out->lanes_per_run = 1;
        out->comps_per_lane = static_cast<int32_t>(n->h.n_comps);
        out->family = 5;
    }
    csmc::IsParams ip = base_params(n, q, seed, first_run, n_runs);
    ip.slab_bytes = L.slab;
    ip.s.flags = flags ? flags : n->d_is_flags;
    ip.s.values = values;
    ip.s.steps = steps;
    ip.logw = logw;
    ip.wvals = n->d_wvals;
    if (coded) {
        rc = theta_cache_for(n, params, st);
        if (rc) return rc;
        ip.theta_cache = n->d_theta_cache;
        ip.cache_mask = kThetaCacheEntries - 1;
        ip.cache_gen = n->theta_gen;
    }
    CK(cudaEventRecord(n->ev0, st), "cudaEventRecord");
    rc = coded ? csmc::is_coded_launch(L.slots, n->is_all_grouped, ip, L.grid, L.block, L.smem, st)
               : csmc::is_launch(n->is_tc, false, L.slots, L.loc8, ip, L.grid, L.block, L.smem, st);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "importance-sampling kernel launch");
    CK(cudaEventRecord(n->ev1, st), "cudaEventRecord");
    reduce_weights<<<csmc::kReduceBlocks, 256, 0, st>>>(n->d_wvals, n_runs, n->d_partials);
    unsigned long long sc[CSMC_SCRATCH_WORDS];
    std::vector<double> part(2 * csmc::kReduceBlocks);
    CK(cudaMemcpyAsync(sc, n->d_scratch, sizeof sc, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CK(cudaMemcpyAsync(part.data(), n->d_partials, part.size() * sizeof(double), cudaMemcpyDeviceToHost, st),
       "cudaMemcpyAsync");
    CK(cudaStreamSynchronize(st), "importance-sampling kernel");
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, n->ev0, n->ev1), "cudaEventElapsedTime");
    out->kernel_ms = ms;
    out->hits = sc[1];
    out->steps = sc[2];
    out->capped = sc[3];
    for (int b = 0; b < csmc::kReduceBlocks; ++b) {
        out->sum += part[2 * b];
        out->sum_sq += part[2 * b + 1];
    }
    out->estimate = out->sum / static_cast<double>(n_runs);
    return CSMC_OK;
}

int csmc_is_trace(csmc_net *n, const csmc_query *q, const void *params, uint64_t seed, uint64_t first_run,
                  const uint64_t *runs, const float *weights, const uint64_t *row_offset, uint64_t n_list, void *rows,
                  uint64_t rows_cap, void *stream) {
    if (!n || !q || !params || !runs || !weights || !row_offset || !rows) return fail(CSMC_ERR_ARG, "null argument");
    int rc = check_query(n, q);
    if (rc) return rc;
    if (n_list == 0) return CSMC_OK;
    CK(cudaSetDevice(n->device), "cudaSetDevice");
    rc = ensure_is_buffers(n, 1);
    if (rc) return rc;
    Launch L;
    rc = plan_is(n, true, n_list, L);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CK(cudaMemcpyAsync(n->d_mlp, params, sizeof(csmc::MlpParams), cudaMemcpyHostToDevice, st), "upload proposal");
    CK(cudaMemsetAsync(n->d_scratch, 0, CSMC_SCRATCH_WORDS * sizeof(unsigned long long), st), "cudaMemsetAsync");
    csmc::IsParams ip = base_params(n, q, seed, first_run, n_list);
    ip.slab_bytes = L.slab;
    ip.trace_runs = runs;
    ip.trace_w = weights;
    ip.row_offset = row_offset;
    ip.rows = static_cast<csmc::MlpRow *>(rows);
    ip.rows_cap = rows_cap;
    rc = csmc::is_launch(n->is_tc, true, L.slots, L.loc8, ip, L.grid, L.block, L.smem, st);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "replay kernel launch");
    unsigned long long sc[CSMC_SCRATCH_WORDS];
    CK(cudaMemcpyAsync(sc, n->d_scratch, sizeof sc, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CK(cudaStreamSynchronize(st), "replay kernel");
    if (sc[4]) return fail(CSMC_ERR_LIMIT, std::to_string(sc[4]) + " replay rows fall beyond the row buffer");
    return CSMC_OK;
}

}  // extern "C"

namespace {

constexpr int kGradFloats = CSMC_MLP_HID * CSMC_MLP_IN + CSMC_MLP_HID * CSMC_MLP_HID + 3 * CSMC_MLP_HID + 1;
static_assert(kGradFloats == CSMC_MLP_GRAD_FLOATS, "gradient layout of include/csmc.h");

// Sums the per-CTA gradient partials of mlp_tc_kernel<1> into the gradient
// (layout w1[64][16], b1[64], w2[64][64], b2[64], w3[64], b3; one thread per
// entry, CTAs in order, FP64) and the per-CTA objectives into J.  A CTA's
// partial block holds D4 = [dZ2 | dZ1]^T . [H1 | X | 1] (128 rows of 96:
// row k < 64 is output unit k of layer 2, row 64 + j is unit j of layer 1;
// columns 0..63 H1, 64..79 X, 80 the bias input), then dw3[64] and db3.
__global__ void reduce_mlp_partials(const float *partials, const double *objective, int grid, int pf, float *grad,
                                    double *J) {
    constexpr int H = CSMC_MLP_HID, I = CSMC_MLP_IN, N4 = 96;
    const int k = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (k < kGradFloats) {
        int src;
        if (k < H * I) src = (64 + k / I) * N4 + 64 + k % I;                       // dW1[j][i]
        else if (k < H * I + H) src = (64 + (k - H * I)) * N4 + 80;               // db1[j]
        else if (k < H * I + H + H * H) src = ((k - H * I - H) / H) * N4 + (k - H * I - H) % H;  // dW2[k][j]
        else if (k < H * I + 2 * H + H * H) src = (k - H * I - H - H * H) * N4 + 80;             // db2[k]
        else if (k < H * I + 3 * H + H * H) src = 128 * N4 + (k - H * I - 2 * H - H * H);        // dw3[k]
        else src = 128 * N4 + 64;                                                                // db3
        double acc = 0.0;
        for (int c = 0; c < grid; ++c) acc = csmc::d_add(acc, static_cast<double>(partials[c * pf + src]));
        grad[k] = static_cast<float>(acc);
    }
    if (k == 0) {
        double s = 0.0;
        for (int c = 0; c < grid; ++c) s = csmc::d_add(s, objective[c]);
        *J = s;
    }
}

// FP32 master vector -> the BF16 parameter block, the host packing's layout
// (w1 and w2 rounded to BF16, biases and the output layer FP32, padding
// zero); one thread per entry.
__global__ void mlp_pack_params(const float *x, csmc::MlpParams *P) {
    constexpr int H = CSMC_MLP_HID, I = CSMC_MLP_IN;
    const int k = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (k < H * I) (&P->w1[0][0])[k] = csmc::f_to_bf16(x[k]);
    else if (k < H * I + H) P->b1[k - H * I] = x[k];
    else if (k < H * I + H + H * H) (&P->w2[0][0])[k - H * I - H] = csmc::f_to_bf16(x[k]);
    else if (k < H * I + 2 * H + H * H) P->b2[k - H * I - H - H * H] = x[k];
    else if (k < H * I + 3 * H + H * H) P->w3[k - H * I - 2 * H - H * H] = x[k];
    else if (k < kGradFloats) P->b3 = x[k];
    else if (k < kGradFloats + 3) P->pad[k - kGradFloats] = 0.0f;
}

// One Adam ascent step per entry (csmc_mlp_adam's formulas, every operation
// an IEEE double operation rounded to nearest, x rounded to FP32).
__global__ void mlp_adam_ascend(float *x, double *m, double *v, const float *g, double lr, double c1, double c2) {
    constexpr double b1 = 0.9, b2 = 0.999, eps = 1e-8;
    const int k = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= kGradFloats) return;
    const double gi = static_cast<double>(g[k]);
    const double mk = csmc::d_add(csmc::d_mul(b1, m[k]), csmc::d_mul(1.0 - b1, gi));
    const double vk = csmc::d_add(csmc::d_mul(b2, v[k]), csmc::d_mul(csmc::d_mul(1.0 - b2, gi), gi));
    m[k] = mk;
    v[k] = vk;
    const double mh = csmc::d_div(mk, c1), vh = csmc::d_div(vk, c2);
    const double up = csmc::d_div(csmc::d_mul(lr, mh), csmc::d_add(csmc::d_sqrt(vh), eps));
    x[k] = static_cast<float>(csmc::d_add(static_cast<double>(x[k]), up));
}

// Device buffers of the proposal-network kernels, one set per device, kept
// for the life of the process (allocating per call would hand the memory
// back to the driver at every synchronisation); a call holds the set's lock
// until its stream has drained.
struct MlpDevScratch {
    std::mutex mu;
    csmc::MlpParams *P = nullptr;
    float *partials = nullptr;
    double *objective = nullptr;
    int *error = nullptr;
    float *grad = nullptr;
    double *J = nullptr;
    float *x = nullptr;         // Adam: master vector
    double *moments = nullptr;  // Adam: m, then v
    double *Js = nullptr;       // Adam: J at the first and the last step
    int grid_cap = 0;
};

MlpDevScratch &mlp_scratch(int dev) {
    static MlpDevScratch sets[64];
    return sets[dev & 63];
}

int mlp_scratch_ensure(MlpDevScratch &m, int grid) {
    if (m.P && grid <= m.grid_cap) return CSMC_OK;
    cudaFree(m.P);
    cudaFree(m.partials);
    cudaFree(m.objective);
    cudaFree(m.error);
    cudaFree(m.grad);
    cudaFree(m.J);
    cudaFree(m.x);
    cudaFree(m.moments);
    cudaFree(m.Js);
    m.x = nullptr;
    m.moments = nullptr;
    m.Js = nullptr;
    m.P = nullptr;
    m.partials = nullptr;
    m.objective = nullptr;
    m.error = nullptr;
    m.grad = nullptr;
    m.J = nullptr;
    m.grid_cap = 0;
    const size_t pf = static_cast<size_t>(csmc::mlp_tc_partial_floats());
    CK(cudaMalloc(&m.P, sizeof(csmc::MlpParams)), "cudaMalloc(proposal network)");
    CK(cudaMalloc(&m.partials, grid * pf * sizeof(float)), "cudaMalloc(gradient partials)");
    CK(cudaMalloc(&m.objective, grid * sizeof(double)), "cudaMalloc(objective partials)");
    CK(cudaMalloc(&m.error, sizeof(int)), "cudaMalloc(error flag)");
    CK(cudaMalloc(&m.grad, kGradFloats * sizeof(float)), "cudaMalloc(gradient)");
    CK(cudaMalloc(&m.J, sizeof(double)), "cudaMalloc(objective)");
    CK(cudaMalloc(&m.x, kGradFloats * sizeof(float)), "cudaMalloc(Adam master vector)");
    CK(cudaMalloc(&m.moments, 2 * kGradFloats * sizeof(double)), "cudaMalloc(Adam moments)");
    CK(cudaMalloc(&m.Js, 2 * sizeof(double)), "cudaMalloc(Adam objectives)");
    m.grid_cap = grid;
    return CSMC_OK;
}

int mlp_common(int mode, const void *params, const void *rows, uint64_t n_rows, float *theta, float *grad,
               double *objective, void *stream) {
    if (!params || (!rows && n_rows)) return fail(CSMC_ERR_ARG, "null argument");
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev), "cudaGetDevice");
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "device attribute");
    const uint64_t tiles = (n_rows + 127) / 128;
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(tiles, sms)));
    const int pf = csmc::mlp_tc_partial_floats();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MlpDevScratch &m = mlp_scratch(dev);
    std::lock_guard<std::mutex> lock(m.mu);
    int rc = mlp_scratch_ensure(m, sms);
    if (rc) return rc;
    CK(cudaMemsetAsync(m.error, 0, sizeof(int), st), "cudaMemsetAsync");
    CK(cudaMemcpyAsync(m.P, params, sizeof(csmc::MlpParams), cudaMemcpyHostToDevice, st), "upload proposal");
    rc = csmc::mlp_tc_launch(mode, static_cast<const csmc::MlpRow *>(rows), n_rows, m.P, theta, m.partials,
                             m.objective, m.error, grid, st);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "tensor-core kernel launch");
    int err = 0;
    double J = 0.0;
    CK(cudaMemcpyAsync(&err, m.error, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    if (mode == 1) {
        reduce_mlp_partials<<<(kGradFloats + 255) / 256, 256, 0, st>>>(m.partials, m.objective, grid, pf, m.grad,
                                                                        m.J);
        CK(cudaGetLastError(), "gradient reduction launch");
        CK(cudaMemcpyAsync(grad, m.grad, kGradFloats * sizeof(float), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        CK(cudaMemcpyAsync(&J, m.J, sizeof(double), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    }
    CK(cudaStreamSynchronize(st), "tensor-core kernel");
    if (err) return fail(CSMC_ERR_TIMEOUT, "tensor-core kernel: a bounded wait for the MMA units gave up");
    if (mode == 1 && objective) *objective = J;
    return CSMC_OK;
}

int mlp_adam(const void *rows, uint64_t n_rows, int32_t steps, double lr, float *x, double *mom1, double *mom2,
             int32_t *t, double *j_first, double *j_last, void *stream) {
    if (!x || !mom1 || !mom2 || !t || (!rows && n_rows)) return fail(CSMC_ERR_ARG, "null argument");
    if (steps < 1 || *t < 0 || *t > INT32_MAX - steps) return fail(CSMC_ERR_ARG, "Adam: steps must be positive");
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev), "cudaGetDevice");
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "device attribute");
    const uint64_t tiles = (n_rows + 127) / 128;
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(tiles, sms)));
    const int pf = csmc::mlp_tc_partial_floats();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MlpDevScratch &m = mlp_scratch(dev);
    std::lock_guard<std::mutex> lock(m.mu);
    int rc = mlp_scratch_ensure(m, sms);
    if (rc) return rc;
    const size_t xb = kGradFloats * sizeof(float), mb = kGradFloats * sizeof(double);
    CK(cudaMemsetAsync(m.error, 0, sizeof(int), st), "cudaMemsetAsync");
    CK(cudaMemcpyAsync(m.x, x, xb, cudaMemcpyHostToDevice, st), "upload master vector");
    CK(cudaMemcpyAsync(m.moments, mom1, mb, cudaMemcpyHostToDevice, st), "upload moments");
    CK(cudaMemcpyAsync(m.moments + kGradFloats, mom2, mb, cudaMemcpyHostToDevice, st), "upload moments");
    constexpr int kThreads = 256, kBlocks = (kGradFloats + 3 + kThreads - 1) / kThreads;
    int32_t tt = *t;
    for (int32_t s = 0; s < steps; ++s) {
        mlp_pack_params<<<kBlocks, kThreads, 0, st>>>(m.x, m.P);
        CK(cudaGetLastError(), "parameter packing launch");
        rc = csmc::mlp_tc_launch(1, static_cast<const csmc::MlpRow *>(rows), n_rows, m.P, nullptr, m.partials,
                                 m.objective, m.error, grid, st);
        if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "tensor-core kernel launch");
        reduce_mlp_partials<<<(kGradFloats + 255) / 256, 256, 0, st>>>(m.partials, m.objective, grid, pf, m.grad,
                                                                        m.Js + (s == 0 ? 0 : 1));
        CK(cudaGetLastError(), "gradient reduction launch");
        ++tt;
        const double c1 = 1.0 - std::pow(0.9, static_cast<double>(tt));
        const double c2 = 1.0 - std::pow(0.999, static_cast<double>(tt));
        mlp_adam_ascend<<<kBlocks, kThreads, 0, st>>>(m.x, m.moments, m.moments + kGradFloats, m.grad, lr, c1, c2);
        CK(cudaGetLastError(), "Adam step launch");
    }
    int err = 0;
    double Js[2] = {0.0, 0.0};
    CK(cudaMemcpyAsync(&err, m.error, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CK(cudaMemcpyAsync(Js, m.Js, sizeof Js, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CK(cudaMemcpyAsync(x, m.x, xb, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CK(cudaMemcpyAsync(mom1, m.moments, mb, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CK(cudaMemcpyAsync(mom2, m.moments + kGradFloats, mb, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CK(cudaStreamSynchronize(st), "Adam steps");
    if (err) return fail(CSMC_ERR_TIMEOUT, "tensor-core kernel: a bounded wait for the MMA units gave up");
    *t = tt;
    if (j_first) *j_first = Js[0];
    if (j_last) *j_last = steps == 1 ? Js[0] : Js[1];
    return CSMC_OK;
}

}  // namespace

extern "C" {

int csmc_mlp_adam(const void *rows, uint64_t n_rows, int32_t steps, double lr, float *x, double *m, double *v,
                  int32_t *t, double *j_first, double *j_last, void *stream) {
    return mlp_adam(rows, n_rows, steps, lr, x, m, v, t, j_first, j_last, stream);
}

int csmc_mlp_forward(const void *params, const void *rows, uint64_t n_rows, float *theta, void *stream) {
    if (!theta && n_rows) return fail(CSMC_ERR_ARG, "null argument");
    return mlp_common(0, params, rows, n_rows, theta, nullptr, nullptr, stream);
}

int csmc_mlp_grad(const void *params, const void *rows, uint64_t n_rows, float *grad, double *objective,
                  void *stream) {
    if (!grad) return fail(CSMC_ERR_ARG, "null argument");
    return mlp_common(1, params, rows, n_rows, nullptr, grad, objective, stream);
}

}  // extern "C"
