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
#include <cstring>
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
    int grid = 0, block = 128;
    size_t smem = 0;
    bool slots = false, loc8 = false;
};

int plan_is(const csmc_net *n, bool trace, uint64_t n_runs, Launch &L) {
    const csmc_net_header &h = n->h;
    L.slots = h.max_edges_per_loc >= 2;
    L.loc8 = h.max_locs_per_comp <= 256;
    const size_t per = csmc::serial_state_bytes_per_thread(h.n_comps, h.n_vars, h.n_rate_prog, L.slots, L.loc8);
    L.smem = n->bytes + csmc::is_mlp_smem_bytes() + (n->is_tc ? csmc::is_stage_bytes(L.block) : 0) +
             ((per * L.block + 15) & ~static_cast<size_t>(15));
    int max_smem = 0, sms = 0, ctas = 0;
    CK(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, n->device), "device attribute");
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n->device), "device attribute");
    if (L.smem > static_cast<size_t>(max_smem))
        return fail(CSMC_ERR_LIMIT, "importance sampling needs the network, the proposal network and the run state "
                                    "of 128 runs in shared memory (" + std::to_string(L.smem) + " bytes)");
    int rc = csmc::is_max_active_ctas(n->is_tc, trace, L.slots, L.loc8, L.block, L.smem, &ctas);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "occupancy query");
    if (ctas < 1) return fail(CSMC_ERR_LIMIT, "importance-sampling kernel cannot be resident");
    uint64_t grid = static_cast<uint64_t>(sms) * ctas;
    const uint64_t needed = (n_runs + L.block - 1) / L.block;
    if (grid > needed) grid = needed;
    L.grid = static_cast<int>(grid);
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
    ip.mlp = n->d_mlp;
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
    out->lanes_per_run = 1;
    out->comps_per_lane = static_cast<int32_t>(n->h.n_comps);
    out->runs_per_cta = 128;
    out->family = 3;
    if (n_runs == 0) return CSMC_OK;
    CK(cudaSetDevice(n->device), "cudaSetDevice");
    rc = ensure_is_buffers(n, n_runs);
    if (rc) return rc;
    Launch L;
    rc = plan_is(n, false, n_runs, L);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CK(cudaMemcpyAsync(n->d_mlp, params, sizeof(csmc::MlpParams), cudaMemcpyHostToDevice, st), "upload proposal");
    CK(cudaMemsetAsync(n->d_scratch, 0, CSMC_SCRATCH_WORDS * sizeof(unsigned long long), st), "cudaMemsetAsync");
    csmc::IsParams ip = base_params(n, q, seed, first_run, n_runs);
    ip.s.flags = flags ? flags : n->d_is_flags;
    ip.s.values = values;
    ip.s.steps = steps;
    ip.logw = logw;
    ip.wvals = n->d_wvals;
    CK(cudaEventRecord(n->ev0, st), "cudaEventRecord");
    rc = csmc::is_launch(n->is_tc, false, L.slots, L.loc8, ip, L.grid, L.block, L.smem, st);
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
                  void *stream) {
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
    ip.trace_runs = runs;
    ip.trace_w = weights;
    ip.row_offset = row_offset;
    ip.rows = static_cast<csmc::MlpRow *>(rows);
    rc = csmc::is_launch(n->is_tc, true, L.slots, L.loc8, ip, L.grid, L.block, L.smem, st);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "replay kernel launch");
    CK(cudaStreamSynchronize(st), "replay kernel");
    return CSMC_OK;
}

}  // extern "C"

namespace {

struct MlpScratch {  // per call, stream-ordered
    csmc::MlpParams *P = nullptr;
    float *partials = nullptr;
    double *objective = nullptr;
    int *error = nullptr;
};

int mlp_common(int mode, const void *params, const void *rows, uint64_t n_rows, float *theta, float *grad,
               double *objective, void *stream) {
    if (!params || (!rows && n_rows)) return fail(CSMC_ERR_ARG, "null argument");
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev), "cudaGetDevice");
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "device attribute");
    const uint64_t tiles = (n_rows + 127) / 128;
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(tiles, sms)));
    const size_t pf = static_cast<size_t>(csmc::mlp_tc_partial_floats());
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MlpScratch m;
    CK(cudaMallocAsync(&m.P, sizeof(csmc::MlpParams), st), "cudaMallocAsync");
    CK(cudaMallocAsync(&m.partials, grid * pf * sizeof(float), st), "cudaMallocAsync");
    CK(cudaMallocAsync(&m.objective, grid * sizeof(double), st), "cudaMallocAsync");
    CK(cudaMallocAsync(&m.error, sizeof(int), st), "cudaMallocAsync");
    CK(cudaMemsetAsync(m.error, 0, sizeof(int), st), "cudaMemsetAsync");
    CK(cudaMemcpyAsync(m.P, params, sizeof(csmc::MlpParams), cudaMemcpyHostToDevice, st), "upload proposal");
    int rc = csmc::mlp_tc_launch(mode, static_cast<const csmc::MlpRow *>(rows), n_rows, m.P, theta, m.partials,
                                 m.objective, m.error, grid, st);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "tensor-core kernel launch");
    int err = 0;
    std::vector<float> part(mode == 1 ? grid * pf : 0);
    std::vector<double> obj(mode == 1 ? grid : 0);
    CK(cudaMemcpyAsync(&err, m.error, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    if (mode == 1) {
        CK(cudaMemcpyAsync(part.data(), m.partials, part.size() * sizeof(float), cudaMemcpyDeviceToHost, st),
           "cudaMemcpyAsync");
        CK(cudaMemcpyAsync(obj.data(), m.objective, obj.size() * sizeof(double), cudaMemcpyDeviceToHost, st),
           "cudaMemcpyAsync");
    }
    cudaFreeAsync(m.P, st);
    cudaFreeAsync(m.partials, st);
    cudaFreeAsync(m.objective, st);
    cudaFreeAsync(m.error, st);
    CK(cudaStreamSynchronize(st), "tensor-core kernel");
    if (err) return fail(CSMC_ERR_TIMEOUT, "tensor-core kernel: a bounded wait for the MMA units gave up");
    if (mode == 1) {
        // gradient layout: w1[64][16], b1[64], w2[64][64], b2[64], w3[64], b3
        constexpr int H = CSMC_MLP_HID, I = CSMC_MLP_IN, N4 = 96;
        std::vector<double> acc(H * I + H + H * H + H + H + 1, 0.0);
        double J = 0.0;
        for (int c = 0; c < grid; ++c) {
            const float *q = part.data() + c * pf;
            for (int k = 0; k < H; ++k) {
                for (int j = 0; j < H; ++j) acc[H * I + H + k * H + j] += q[k * N4 + j];  // dW2[k][j]
                acc[H * I + H + H * H + k] += q[k * N4 + 80];                             // db2[k]
            }
            for (int j = 0; j < H; ++j) {
                for (int i = 0; i < I; ++i) acc[j * I + i] += q[(64 + j) * N4 + 64 + i];  // dW1[j][i]
                acc[H * I + j] += q[(64 + j) * N4 + 80];                                // db1[j]
            }
            for (int k = 0; k < H; ++k) acc[H * I + H + H * H + H + k] += q[128 * N4 + k];  // dw3[k]
            acc[H * I + H + H * H + H + H] += q[128 * N4 + 64];                            // db3
            J += obj[c];
        }
        for (size_t i = 0; i < acc.size(); ++i) grad[i] = static_cast<float>(acc[i]);
        if (objective) *objective = J;
    }
    return CSMC_OK;
}

}  // namespace

extern "C" {

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
