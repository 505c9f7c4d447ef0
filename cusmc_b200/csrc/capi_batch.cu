// C ABI of batches (many (network, query) jobs in one persistent launch of
// the batch kernel, sim_batch.cuh) and of the launch-plan autotuners.
#include "../../include/csmc.h"
#include "capi_internal.h"
#include "include/csmc_net.h"
#include "kernels/reduce.cuh"
#include "kernels/sim.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

// Jobs whose networks have at least this many components (and at most
// CSMC_BATCH_GROUP_MAX_COMPS) run one warp per run by default.
constexpr uint32_t kDefaultGroupMinComps = 128;
// Counter words before the per-job counters: the two run queues.
constexpr size_t kQueueWords = 2;

struct csmc_batch {
    int device = 0;
    int n_jobs = 0;
    bool verify = false;
    std::vector<csmc_net *> nets;
    std::vector<csmc_query> qs;
    std::vector<uint64_t> seeds, first_runs, n_runs;
    std::vector<double> cost;          // estimated device cost of one run, per job
    std::vector<int> order;            // job-table position -> job: warp-per-run jobs first, each part by cost
    std::vector<char> group;           // per job: simulated one warp per run
    int n_group = 0;                   // warp-per-run jobs
    uint32_t group_min_comps = kDefaultGroupMinComps;  // networks this large run one warp per run (0: none do)
    int group_k = 0;                   // components per lane of the warp-per-run jobs
    uint32_t group_stride = 0;         // shared memory of one warp-per-run run state
    std::vector<uint64_t> out_off;     // per job: first run's index in the output buffers
    std::vector<uint64_t> fs_off;      // per job: offset of its final states (words)
    uint64_t total_runs = 0;
    uint32_t max_v = 0, max_p = 0, max_c = 0;  // over the thread-per-run jobs
    csmc::BatchJob *d_jobs = nullptr;  // in job-table order
    uint8_t *d_flags = nullptr;
    double *d_values = nullptr;
    uint32_t *d_steps = nullptr;
    uint64_t *d_digests = nullptr;
    uint32_t *d_final = nullptr;
    unsigned long long *d_counters = nullptr;  // [0] thread-per-run queue, [1] warp-per-run queue, then 4 words per job-table position
    double *d_partials = nullptr;              // 2 * kReduceBlocks per job-table position
    unsigned long long *h_counters = nullptr;  // pinned copies
    double *h_partials = nullptr;
    uint8_t *d_state = nullptr;
    size_t state_bytes = 0;
    int block = 128, ctas_per_sm = 0, grid = 0;
    uint32_t state_stride = 0;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

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

// Per-job value sums, one block row per run-space position (the arithmetic
// of csmc_run's reduction, so each job's sums carry the same bits).
__global__ void reduce_jobs(const csmc::BatchJob *jobs, double *partials) {
    const csmc::BatchJob &J = jobs[blockIdx.y];
    double *out = partials + (static_cast<size_t>(blockIdx.y) * csmc::kReduceBlocks + blockIdx.x) * 2;
    csmc::reduce_block(J.values, J.n_runs, blockIdx.x, out);
}

int check_query(const csmc_net *n, const csmc_query *q) {
    if (q->kind != CSMC_QUERY_LOCATION && q->kind != CSMC_QUERY_VARIABLE) return fail(CSMC_ERR_ARG, "bad query kind");
    if (q->kind == CSMC_QUERY_VARIABLE && (q->var_id < 0 || static_cast<uint32_t>(q->var_id) >= n->h.n_vars))
        return fail(CSMC_ERR_ARG, "query variable id " + std::to_string(q->var_id) + " out of range");
    return CSMC_OK;
}

void drop_graph(csmc_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
}

// Which jobs run one warp per run (networks of group_min_comps ..
// CSMC_BATCH_GROUP_MAX_COMPS components), the job-table order (those jobs
// first, each part by falling cost), the lanes' component count and the
// state sizes of both parts.
void assign_modes(csmc_batch *b) {
    b->group.assign(b->n_jobs, 0);
    b->n_group = 0;
    b->max_v = b->max_p = b->max_c = 0;
    uint32_t gmax_c = 0, gmax_vp = 0;
    for (int j = 0; j < b->n_jobs; ++j) {
        const csmc_net_header &h = b->nets[j]->h;
        const bool g = b->group_min_comps > 0 && h.n_comps >= b->group_min_comps &&
                       h.n_comps <= CSMC_BATCH_GROUP_MAX_COMPS;
        b->group[j] = g;
        if (g) {
            ++b->n_group;
            gmax_c = std::max(gmax_c, h.n_comps);
            gmax_vp = std::max(gmax_vp, h.n_vars + h.n_rate_prog);
        } else {
            b->max_v = std::max(b->max_v, h.n_vars);
            b->max_p = std::max(b->max_p, h.n_rate_prog);
            b->max_c = std::max(b->max_c, h.n_comps);
        }
    }
    b->group_k = gmax_c == 0 ? 0 : gmax_c <= 128 ? 4 : gmax_c <= 256 ? 8 : 16;
    b->group_stride = b->n_group ? csmc::group_state_stride(gmax_vp, 0, 32, b->group_k) : 0;
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
        if (b->group[x] != b->group[y]) return b->group[x] > b->group[y];
        return b->cost[x] > b->cost[y];
    });
}

// Runs of the thread-per-run part and of the warp-per-run part.
void part_totals(const csmc_batch *b, const std::vector<uint64_t> &runs, uint64_t *thread_runs,
                 uint64_t *group_runs) {
    *thread_runs = *group_runs = 0;
    for (int j = 0; j < b->n_jobs; ++j) (b->group[j] ? *group_runs : *thread_runs) += runs[j];
}

// Job table in job-table order for the given per-job run counts (each part
// numbers its runs from 0); step_cap (0: none) limits every run's race
// steps (autotuner probes).
std::vector<csmc::BatchJob> build_table(const csmc_batch *b, const std::vector<uint64_t> &runs, uint64_t step_cap = 0) {
    std::vector<csmc::BatchJob> t(b->n_jobs);
    uint64_t begin[2] = {0, 0};
    for (int k = 0; k < b->n_jobs; ++k) {
        const int j = b->order[k];
        const csmc_net *n = b->nets[j];
        const csmc_query &q = b->qs[j];
        csmc::BatchJob &J = t[k];
        std::memset(&J, 0, sizeof J);
        J.net = csmc::layout_of(n->h);
        J.blob = n->d_blob;
        J.run_begin = begin[b->group[j] ? 1 : 0];
        J.n_runs = runs[j];
        J.first_run = b->first_runs[j];
        J.seed = b->seeds[j];
        J.max_steps = q.max_steps ? q.max_steps : 10000000ull;
        if (step_cap && J.max_steps > step_cap) J.max_steps = step_cap;
        J.threshold = q.threshold;
        J.horizon = static_cast<float>(q.horizon);
        J.loc_mode = q.kind == CSMC_QUERY_LOCATION;
        J.var_id = q.var_id;
        J.is_max = q.is_max;
        J.flags = b->d_flags + b->out_off[j];
        J.values = b->d_values + b->out_off[j];
        J.steps = b->d_steps + b->out_off[j];
        J.digests = b->d_digests ? b->d_digests + b->out_off[j] : nullptr;
        J.final_state = b->d_final ? b->d_final + b->fs_off[j] : nullptr;
        J.counters = b->d_counters + kQueueWords + 4 * static_cast<size_t>(k);
        begin[b->group[j] ? 1 : 0] += runs[j];
    }
    return t;
}

int upload_table(csmc_batch *b, const std::vector<uint64_t> &runs, uint64_t step_cap = 0) {
    const std::vector<csmc::BatchJob> t = build_table(b, runs, step_cap);
    CK(cudaMemcpy(b->d_jobs, t.data(), t.size() * sizeof(csmc::BatchJob), cudaMemcpyHostToDevice),
       "cudaMemcpy(job table)");
    return CSMC_OK;
}

size_t launch_smem(const csmc_batch *b, int block) {
    return csmc::batch_smem_bytes(b->n_jobs, b->n_group ? b->group_stride : 0u, block);
}

// Grid and state slabs for the current geometry.
int configure(csmc_batch *b) {
    int ctas = 0, sms = 0;
    const size_t smem = launch_smem(b, b->block);
    int rc = csmc::batch_max_active_ctas(b->verify, b->n_group ? b->group_k : 0, b->block, smem, &ctas);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "occupancy query");
    if (ctas < 1) return fail(CSMC_ERR_LIMIT, "batch kernel cannot be resident");
    if (b->ctas_per_sm > 0) ctas = std::min(ctas, b->ctas_per_sm);
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "cudaDeviceGetAttribute");
    uint64_t grid = static_cast<uint64_t>(sms) * ctas;
    uint64_t thread_runs = 0, group_runs = 0;
    part_totals(b, b->n_runs, &thread_runs, &group_runs);
    const uint64_t warps = b->block / 32;
    const uint64_t needed = (thread_runs + b->block - 1) / b->block + (group_runs + warps - 1) / warps;
    grid = std::max<uint64_t>(1, std::min(grid, needed));
    const size_t per = b->n_group == b->n_jobs ? 0 : csmc::batch_state_bytes_per_thread(b->max_c, b->max_v, b->max_p);
    b->state_stride = static_cast<uint32_t>((per * b->block + 15) & ~static_cast<size_t>(15));
    const size_t need = std::max<size_t>(16, grid * static_cast<size_t>(b->state_stride));
    if (need > b->state_bytes) {
        cudaFree(b->d_state);
        b->d_state = nullptr;
        b->state_bytes = 0;
        CK(cudaMalloc(&b->d_state, need), "cudaMalloc(batch run state)");
        b->state_bytes = need;
    }
    b->grid = static_cast<int>(grid);
    drop_graph(b);
    return CSMC_OK;
}

// The launch sequence: no allocation, no synchronisation (capturable).
int launch_impl(csmc_batch *b, cudaStream_t st, const std::vector<uint64_t> &runs) {
    const size_t words = kQueueWords + 4 * static_cast<size_t>(b->n_jobs);
    CK(cudaMemsetAsync(b->d_counters, 0, words * sizeof(unsigned long long), st), "cudaMemsetAsync(batch counters)");
    uint64_t thread_runs = 0, group_runs = 0;
    part_totals(b, runs, &thread_runs, &group_runs);
    csmc::BatchParams p{};
    p.jobs = b->d_jobs;
    p.n_jobs = static_cast<uint32_t>(b->n_jobs);
    p.state_stride = b->state_stride;
    p.total_runs = thread_runs;
    p.queue = b->d_counters;
    p.state = b->d_state;
    p.max_vars = b->max_v;
    p.max_rate_prog = b->max_p;
    p.max_comps = b->max_c;
    p.n_group_jobs = static_cast<uint32_t>(b->n_group);
    p.group_runs = group_runs;
    p.group_queue = b->n_group ? b->d_counters + 1 : nullptr;
    p.group_stride = b->group_stride;
    p.group_k = static_cast<uint32_t>(b->group_k);
    int rc = csmc::batch_launch(b->verify, p, b->grid, b->block, st);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "batch kernel launch");
    reduce_jobs<<<dim3(csmc::kReduceBlocks, b->n_jobs), 256, 0, st>>>(b->d_jobs, b->d_partials);
    CK(cudaGetLastError(), "reduce launch");
    CK(cudaMemcpyAsync(b->h_counters, b->d_counters, words * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st),
       "cudaMemcpyAsync(batch counters)");
    CK(cudaMemcpyAsync(b->h_partials, b->d_partials,
                       2 * csmc::kReduceBlocks * static_cast<size_t>(b->n_jobs) * sizeof(double), cudaMemcpyDeviceToHost,
                       st),
       "cudaMemcpyAsync(batch sums)");
    return CSMC_OK;
}

void fill_results(const csmc_batch *b, const std::vector<uint64_t> &runs, float ms, csmc_result *outs) {
    for (int k = 0; k < b->n_jobs; ++k) {
        const int j = b->order[k];
        csmc_result &r = outs[j];
        std::memset(&r, 0, sizeof r);
        const unsigned long long *c = b->h_counters + kQueueWords + 4 * static_cast<size_t>(k);
        r.runs = runs[j];
        r.hits = c[0];
        r.steps = c[1];
        r.capped = c[2];
        const double *part = b->h_partials + static_cast<size_t>(k) * 2 * csmc::kReduceBlocks;
        for (int i = 0; i < csmc::kReduceBlocks; ++i) {
            r.sum += part[2 * i];
            r.sum_sq += part[2 * i + 1];
        }
        const csmc_query &q = b->qs[j];
        if (r.runs == 0) r.estimate = 0.0;
        else if (q.kind == CSMC_QUERY_VARIABLE && q.is_estimate) r.estimate = r.sum / static_cast<double>(r.runs);
        else r.estimate = static_cast<double>(r.hits) / static_cast<double>(r.runs);
        r.kernel_ms = ms;
        r.lanes_per_run = b->group[j] ? 32 : 1;
        r.comps_per_lane = b->group[j] ? b->group_k : static_cast<int32_t>(b->nets[j]->h.n_comps);
        r.runs_per_cta = b->group[j] ? b->block / 32 : b->block;
        r.family = 2;
    }
}

// Probe of the batch at the current geometry with the given run counts:
// device time in ms; per-job steps in steps_out (job order).
// Probes cap every run at kProbeSteps race steps, so that a probe costs a
// bounded amount of work even when single runs of a job take seconds.
constexpr uint64_t kProbeSteps = 2000;

int probe(csmc_batch *b, const std::vector<uint64_t> &runs, float *ms, std::vector<uint64_t> *steps_out) {
    int rc = upload_table(b, runs, kProbeSteps);
    if (rc) return rc;
    cudaStream_t st = nullptr;
    CK(cudaEventRecord(b->ev0, st), "cudaEventRecord");
    rc = launch_impl(b, st, runs);
    if (rc) return rc;
    CK(cudaEventRecord(b->ev1, st), "cudaEventRecord");
    CK(cudaStreamSynchronize(st), "batch probe");
    CK(cudaEventElapsedTime(ms, b->ev0, b->ev1), "cudaEventElapsedTime");
    if (steps_out) {  // per job: steps, or 0 when some run hit the probe's cap
        steps_out->assign(b->n_jobs, 0);
        for (int k = 0; k < b->n_jobs; ++k) {
            const unsigned long long *c = b->h_counters + kQueueWords + 4 * static_cast<size_t>(k);
            (*steps_out)[b->order[k]] = c[2] ? 0 : c[1];
        }
    }
    return CSMC_OK;
}

}  // namespace

extern "C" {

int csmc_batch_create(csmc_net *const *nets, const csmc_query *qs, const uint64_t *seeds, const uint64_t *first_runs,
                      const uint64_t *n_runs, int32_t n_jobs, int32_t verify, csmc_batch **out) {
    if (!nets || !qs || !seeds || !n_runs || !out) return fail(CSMC_ERR_ARG, "null argument");
    *out = nullptr;
    if (n_jobs < 1 || n_jobs > CSMC_BATCH_MAX_JOBS)
        return fail(CSMC_ERR_LIMIT, "a batch holds 1 to " + std::to_string(CSMC_BATCH_MAX_JOBS) + " jobs");
    auto b = std::make_unique<csmc_batch>();
    CK(cudaGetDevice(&b->device), "cudaGetDevice");
    b->n_jobs = n_jobs;
    b->verify = verify != 0;
    uint64_t fs_words = 0;
    for (int j = 0; j < n_jobs; ++j) {
        const csmc_net *n = nets[j];
        if (!n) return fail(CSMC_ERR_ARG, "null network handle in job " + std::to_string(j));
        if (n->device != b->device) return fail(CSMC_ERR_ARG, "job " + std::to_string(j) + " is on another device");
        int rc = check_query(n, &qs[j]);
        if (rc) return rc;
        const uint64_t fr = first_runs ? first_runs[j] : 0;
        if (fr + n_runs[j] < fr || fr + n_runs[j] > (1ull << 62)) return fail(CSMC_ERR_ARG, "run range out of bounds");
        if (n->h.n_locs > 0xffffu) return fail(CSMC_ERR_LIMIT, "job " + std::to_string(j) + " has more than 65535 locations");
        b->nets.push_back(nets[j]);
        b->qs.push_back(qs[j]);
        b->seeds.push_back(seeds[j]);
        b->first_runs.push_back(fr);
        b->n_runs.push_back(n_runs[j]);
        b->out_off.push_back(b->total_runs);
        b->fs_off.push_back(fs_words);
        b->total_runs += n_runs[j];
        fs_words += n_runs[j] * (n->h.n_comps + n->h.n_vars);
        // until measured: cost of a run ~ components x horizon
        b->cost.push_back(static_cast<double>(n->h.n_comps) * std::max(1.0, qs[j].horizon));
    }
    b->order.resize(n_jobs);
    std::iota(b->order.begin(), b->order.end(), 0);
    assign_modes(b.get());
    const uint64_t R = std::max<uint64_t>(b->total_runs, 1);
    CK(cudaMalloc(&b->d_jobs, n_jobs * sizeof(csmc::BatchJob)), "cudaMalloc(job table)");
    CK(cudaMalloc(&b->d_flags, R), "cudaMalloc(flags)");
    CK(cudaMalloc(&b->d_values, R * sizeof(double)), "cudaMalloc(values)");
    CK(cudaMalloc(&b->d_steps, R * sizeof(uint32_t)), "cudaMalloc(steps)");
    if (b->verify) {
        CK(cudaMalloc(&b->d_digests, R * sizeof(uint64_t)), "cudaMalloc(digests)");
        CK(cudaMalloc(&b->d_final, std::max<uint64_t>(fs_words, 1) * sizeof(uint32_t)), "cudaMalloc(final states)");
    }
    const size_t counters = kQueueWords + 4 * static_cast<size_t>(n_jobs);
    const size_t partials = 2 * csmc::kReduceBlocks * static_cast<size_t>(n_jobs);
    CK(cudaMalloc(&b->d_counters, counters * sizeof(unsigned long long)), "cudaMalloc(counters)");
    CK(cudaMalloc(&b->d_partials, partials * sizeof(double)), "cudaMalloc(partials)");
    CK(cudaMallocHost(&b->h_counters, counters * sizeof(unsigned long long)), "cudaMallocHost(counters)");
    CK(cudaMallocHost(&b->h_partials, partials * sizeof(double)), "cudaMallocHost(partials)");
    std::memset(b->h_counters, 0, counters * sizeof(unsigned long long));
    std::memset(b->h_partials, 0, partials * sizeof(double));
    CK(cudaEventCreate(&b->ev0), "cudaEventCreate");
    CK(cudaEventCreate(&b->ev1), "cudaEventCreate");
    CK(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking), "cudaStreamCreate");
    int rc = configure(b.get());
    if (rc) return rc;
    rc = upload_table(b.get(), b->n_runs);
    if (rc) return rc;
    *out = b.release();
    return CSMC_OK;
}

int csmc_batch_set_plan(csmc_batch *b, int32_t threads_per_cta, int32_t ctas_per_sm) {
    if (!b) return fail(CSMC_ERR_ARG, "null argument");
    if (threads_per_cta < 32 || threads_per_cta > 128 || threads_per_cta % 32)
        return fail(CSMC_ERR_ARG, "batch plans use 32..128 threads per CTA (multiples of 32)");
    if (ctas_per_sm < 0) return fail(CSMC_ERR_ARG, "negative CTAs per SM");
    CK(cudaSetDevice(b->device), "cudaSetDevice");
    b->block = threads_per_cta;
    b->ctas_per_sm = ctas_per_sm;
    return configure(b);
}

int csmc_batch_plan(const csmc_batch *b, int32_t *threads_per_cta, int32_t *ctas_per_sm) {
    if (!b) return fail(CSMC_ERR_ARG, "null argument");
    if (threads_per_cta) *threads_per_cta = b->block;
    if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
    return CSMC_OK;
}

int csmc_batch_launch(csmc_batch *b, void *stream) {
    if (!b) return fail(CSMC_ERR_ARG, "null argument");
    return launch_impl(b, static_cast<cudaStream_t>(stream), b->n_runs);
}

int csmc_batch_set_group_comps(csmc_batch *b, int32_t min_comps) {
    if (!b) return fail(CSMC_ERR_ARG, "null argument");
    if (min_comps < 0) return fail(CSMC_ERR_ARG, "negative component threshold");
    CK(cudaSetDevice(b->device), "cudaSetDevice");
    b->group_min_comps = static_cast<uint32_t>(min_comps);
    assign_modes(b);
    int rc = configure(b);
    if (rc) return rc;
    return upload_table(b, b->n_runs);
}

int csmc_batch_group_comps(const csmc_batch *b, int32_t *min_comps, int32_t *group_jobs) {
    if (!b) return fail(CSMC_ERR_ARG, "null argument");
    if (min_comps) *min_comps = static_cast<int32_t>(b->group_min_comps);
    if (group_jobs) *group_jobs = b->n_group;
    return CSMC_OK;
}

int csmc_batch_results(const csmc_batch *b, csmc_result *outs) {
    if (!b || !outs) return fail(CSMC_ERR_ARG, "null argument");
    fill_results(b, b->n_runs, 0.0f, outs);
    return CSMC_OK;
}

int csmc_batch_run(csmc_batch *b, int32_t use_graph, void *stream, csmc_result *outs) {
    if (!b || !outs) return fail(CSMC_ERR_ARG, "null argument");
    CK(cudaSetDevice(b->device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (use_graph && !b->exec) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        int rc = launch_impl(b, b->cap, b->n_runs);
        cudaError_t e = cudaStreamEndCapture(b->cap, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            return cuda_fail(e, "cudaGraphInstantiate");
        }
    }
    CK(cudaEventRecord(b->ev0, st), "cudaEventRecord");
    if (use_graph) {
        CK(cudaGraphLaunch(b->exec, st), "cudaGraphLaunch");
    } else {
        int rc = launch_impl(b, st, b->n_runs);
        if (rc) return rc;
    }
    CK(cudaEventRecord(b->ev1, st), "cudaEventRecord");
    CK(cudaStreamSynchronize(st), "batch");
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1), "cudaEventElapsedTime");
    fill_results(b, b->n_runs, ms, outs);
    return CSMC_OK;
}

int csmc_batch_outputs(const csmc_batch *b, int32_t job, uint8_t **flags, double **values, uint32_t **steps,
                       uint64_t **digests, uint32_t **final_state) {
    if (!b) return fail(CSMC_ERR_ARG, "null argument");
    if (job < 0 || job >= b->n_jobs) return fail(CSMC_ERR_ARG, "job index out of range");
    const uint64_t o = b->out_off[job];
    if (flags) *flags = b->d_flags + o;
    if (values) *values = b->d_values + o;
    if (steps) *steps = b->d_steps + o;
    if (digests) *digests = b->d_digests ? b->d_digests + o : nullptr;
    if (final_state) *final_state = b->d_final ? b->d_final + b->fs_off[job] : nullptr;
    return CSMC_OK;
}

int csmc_batch_outputs_host(const csmc_batch *b, int32_t job, uint8_t *flags, double *values, uint32_t *steps,
                            uint64_t *digests, uint32_t *final_state) {
    if (!b) return fail(CSMC_ERR_ARG, "null argument");
    if (job < 0 || job >= b->n_jobs) return fail(CSMC_ERR_ARG, "job index out of range");
    CK(cudaSetDevice(b->device), "cudaSetDevice");
    const uint64_t o = b->out_off[job], n = b->n_runs[job];
    const uint64_t words = n * (b->nets[job]->h.n_comps + b->nets[job]->h.n_vars);
    if (n == 0) return CSMC_OK;
    if (flags) CK(cudaMemcpy(flags, b->d_flags + o, n, cudaMemcpyDeviceToHost), "cudaMemcpy(flags)");
    if (values) CK(cudaMemcpy(values, b->d_values + o, n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy(values)");
    if (steps) CK(cudaMemcpy(steps, b->d_steps + o, n * sizeof(uint32_t), cudaMemcpyDeviceToHost), "cudaMemcpy(steps)");
    if (digests) {
        if (!b->d_digests) return fail(CSMC_ERR_ARG, "the batch was created without verification outputs");
        CK(cudaMemcpy(digests, b->d_digests + o, n * sizeof(uint64_t), cudaMemcpyDeviceToHost), "cudaMemcpy(digests)");
    }
    if (final_state) {
        if (!b->d_final) return fail(CSMC_ERR_ARG, "the batch was created without verification outputs");
        CK(cudaMemcpy(final_state, b->d_final + b->fs_off[job], words * sizeof(uint32_t), cudaMemcpyDeviceToHost),
           "cudaMemcpy(final states)");
    }
    return CSMC_OK;
}

int csmc_batch_autotune(csmc_batch *b, double probe_fraction, int32_t *threads_per_cta, int32_t *ctas_per_sm) {
    if (!b) return fail(CSMC_ERR_ARG, "null argument");
    if (!(probe_fraction > 0.0 && probe_fraction <= 1.0)) return fail(CSMC_ERR_ARG, "probe fraction must be in (0, 1]");
    CK(cudaSetDevice(b->device), "cudaSetDevice");
    std::vector<uint64_t> runs(b->n_jobs);
    for (int j = 0; j < b->n_jobs; ++j)
        runs[j] = b->n_runs[j] ? std::max<uint64_t>(1, static_cast<uint64_t>(b->n_runs[j] * probe_fraction)) : 0;
    const int save_block = b->block, save_ctas = b->ctas_per_sm;
    // 1. measure the cost per run of every job at the current geometry
    std::vector<uint64_t> steps;
    float ms = 0.0f;
    int rc = probe(b, runs, &ms, &steps);
    if (rc) return rc;
    for (int j = 0; j < b->n_jobs; ++j)  // measured cost per run where no probe run was capped
        if (runs[j] && steps[j])
            b->cost[j] = static_cast<double>(steps[j]) / runs[j] * std::max<uint32_t>(1, b->nets[j]->h.n_comps);
    assign_modes(b);
    // 2. geometry: threads per CTA x CTAs per SM
    int best_block = save_block, best_ctas = save_ctas;
    float best_ms = -1.0f;
    for (int block : {64, 128}) {
        int maxc = 0;
        rc = csmc::batch_max_active_ctas(b->verify, b->n_group ? b->group_k : 0, block, launch_smem(b, block), &maxc);
        if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "occupancy query");
        for (int c = maxc; c >= 1 && c >= maxc - 3; --c) {
            b->block = block;
            b->ctas_per_sm = c;
            rc = configure(b);
            if (rc) return rc;
            rc = probe(b, runs, &ms, nullptr);
            if (rc) return rc;
            if (best_ms < 0.0f || ms < best_ms) {
                best_ms = ms;
                best_block = block;
                best_ctas = c;
            }
        }
    }
    b->block = best_block;
    b->ctas_per_sm = best_ctas;
    // 3. which networks run one warp per run, at that geometry
    const uint32_t save_min = b->group_min_comps;
    uint32_t best_min = save_min;
    for (uint32_t m : {0u, 64u, 128u, 256u}) {
        if (m == save_min) continue;
        b->group_min_comps = m;
        assign_modes(b);
        rc = configure(b);
        if (rc) return rc;
        rc = probe(b, runs, &ms, nullptr);
        if (rc) return rc;
        if (ms < best_ms) {
            best_ms = ms;
            best_min = m;
        }
    }
    b->group_min_comps = best_min;
    assign_modes(b);
    rc = configure(b);
    if (rc) return rc;
    rc = upload_table(b, b->n_runs);
    if (rc) return rc;
    if (threads_per_cta) *threads_per_cta = best_block;
    if (ctas_per_sm) *ctas_per_sm = best_ctas;
    return CSMC_OK;
}

void csmc_batch_free(csmc_batch *b) {
    if (!b) return;
    drop_graph(b);
    cudaFree(b->d_jobs);
    cudaFree(b->d_flags);
    cudaFree(b->d_values);
    cudaFree(b->d_steps);
    cudaFree(b->d_digests);
    cudaFree(b->d_final);
    cudaFree(b->d_counters);
    cudaFree(b->d_partials);
    cudaFree(b->d_state);
    cudaFreeHost(b->h_counters);
    cudaFreeHost(b->h_partials);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->cap) cudaStreamDestroy(b->cap);
    delete b;
}

int csmc_autotune(csmc_net *n, const csmc_query *q, uint64_t seed, uint64_t probe_runs, csmc_result *best) {
    if (!n || !q || !best) return fail(CSMC_ERR_ARG, "null argument");
    if (probe_runs == 0) return fail(CSMC_ERR_ARG, "probe_runs must be positive");
    int32_t saved[4] = {n->family, n->lanes, n->comps_per_lane, n->block};
    struct Cand {
        int family, lanes, cpl, block;
    };
    std::vector<Cand> cands;
    const int C = static_cast<int>(n->h.n_comps);
    int G = 1, K = 1;
    if (C <= 32) {
        while (G < C) G <<= 1;
    } else {
        G = 32;
        K = 2;
        while (G * K < C) K <<= 1;
    }
    for (int block : {64, 128}) cands.push_back({4, 1, C, block});
    for (int block : {64, 128}) cands.push_back({1, 1, C, block});
    for (int block : {128, 256}) cands.push_back({0, G, K, block});
    for (int block : {64, 128}) cands.push_back({2, 1, C, block});
    csmc_result r{}, top{};
    bool have = false;
    int32_t pick[4] = {saved[0], saved[1], saved[2], saved[3]};
    for (const Cand &c : cands) {
        if (csmc_set_plan(n, c.family, c.lanes, c.cpl, c.block) != CSMC_OK) continue;
        if (csmc_run(n, q, seed, 0, probe_runs, nullptr, nullptr, nullptr, &r, nullptr) != CSMC_OK) continue;
        if (!have || r.kernel_ms < top.kernel_ms) {
            top = r;
            have = true;
            pick[0] = c.family;
            pick[1] = c.lanes;
            pick[2] = c.cpl;
            pick[3] = c.block;
        }
    }
    if (!have) {
        csmc_set_plan(n, saved[0], saved[1], saved[2], saved[3]);
        return fail(CSMC_ERR_LIMIT, "no plan could run this network");
    }
    int rc = csmc_set_plan(n, pick[0], pick[1], pick[2], pick[3]);
    if (rc) return rc;
    *best = top;
    return CSMC_OK;
}

}  // extern "C"
