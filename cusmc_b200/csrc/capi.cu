// C ABI of libcsmc (include/csmc.h): front end, device network handles,
// launches, result collection, and the reference's smc() report.
#include "../../include/csmc.h"
#include "front/front.h"
#include "include/csmc_net.h"
#include "include/csmc_numeric.h"
#include "kernels/sim.cuh"
#include "kernels/reduce.cuh"
#include "capi_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &m) {
    g_err = m;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(CSMC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(x, what)                          \
    do {                                     \
        cudaError_t e_ = (x);                \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// Lane-group shape for C components: one lane per component up to a warp,
// then a full warp with K components per lane.
void choose_shape(uint32_t C, int &G, int &K) {
    if (C <= 32) {
        G = 1;
        while (static_cast<uint32_t>(G) < C) G <<= 1;
        K = 1;
        return;
    }
    G = 32;
    K = 2;
    while (static_cast<uint32_t>(G * K) < C) K <<= 1;
}

int max_smem_optin(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    return v;
}

// Fills the launch geometry of a plan; returns false when it cannot run.
bool configure_plan(csmc_net *n, int family, int lanes, int cpl, int block, std::string &why) {
    const csmc_net_header &h = n->h;
    const size_t max_smem = static_cast<size_t>(max_smem_optin(n->device));
    if (family == 0) {
        if (!csmc::sim_supported(lanes, cpl) || static_cast<uint64_t>(lanes) * cpl < h.n_comps) {
            why = "unsupported lane-group shape";
            return false;
        }
        if (block <= 0 || block % 32 || block % lanes || block > 256) {
            why = "lane-group plans use 32..256 threads per CTA";
            return false;
        }
        // per-group run state: 48 bytes of scalars, the variables, one
        // inverse rate per rate program (evaluated once per step), the slot
        // masks
        const uint32_t stride = csmc::group_state_stride(h.n_vars, h.n_rate_prog, lanes, cpl);
        const size_t smem = n->bytes + static_cast<size_t>(block / lanes) * stride;
        if (smem > max_smem) {
            why = "network and run state do not fit in shared memory";
            return false;
        }
        n->family = 0;
        n->lanes = lanes;
        n->comps_per_lane = cpl;
        n->block = block;
        n->state_stride = stride;
        n->smem = smem;
        n->state_in_global = false;
        return true;
    }
    if (block <= 0 || block % 32 || block > 128) {
        why = "thread-per-run plans use 32..128 threads per CTA";
        return false;
    }
    if (family == 4) {  // class-coded thread per run (sim_coded.cuh)
        if (!n->classes || h.n_comps < 4 || h.n_comps > 256 || h.max_locs_per_comp > 32) {
            why = "the class-coded plan needs race classes, 4 to 256 components and at most 32 locations per "
                  "automaton";
            return false;
        }
        const csmc::NetLayout L = csmc::layout_of(h);
        const size_t slab = csmc::coded_slab_bytes(h.n_comps, h.n_vars, h.n_rate_prog, n->slots, block, L.n_classes,
                                                   (h.recv_chan_lo | h.recv_chan_hi) != 0);
        if (n->bytes + slab > max_smem) {
            why = "network and run state do not fit in shared memory";
            return false;
        }
        n->family = 4;
        n->lanes = 1;
        n->comps_per_lane = static_cast<int>(h.n_comps);
        n->block = block;
        n->state_stride = static_cast<uint32_t>(slab);
        n->state_in_global = false;
        n->smem = n->bytes + slab;
        return true;
    }
    if (family == 2) {  // network and run state in global memory
        if (h.max_locs_per_comp > 0xffffu || h.n_locs > 0xffffu) {
            why = "more than 65535 locations";
            return false;
        }
        const size_t per = csmc::batch_state_bytes_per_thread(h.n_comps, h.n_vars, h.n_rate_prog);
        n->family = 2;
        n->lanes = 1;
        n->comps_per_lane = static_cast<int>(h.n_comps);
        n->block = block;
        n->state_stride = static_cast<uint32_t>((per * block + 15) & ~static_cast<size_t>(15));
        n->state_in_global = true;
        n->smem = csmc::batch_smem_bytes(1);
        return true;
    }
    if (family != 1) {
        why = "unknown plan family";
        return false;
    }
    if (n->bytes > max_smem) {
        why = "network does not fit in shared memory";
        return false;
    }
    const size_t per_thread = csmc::serial_state_bytes_per_thread(h.n_comps, h.n_vars, h.n_rate_prog, n->slots, n->loc8);
    const size_t slab = (per_thread * block + 15) & ~static_cast<size_t>(15);
    n->family = 1;
    n->lanes = 1;
    n->comps_per_lane = static_cast<int>(h.n_comps);
    n->block = block;
    n->state_stride = static_cast<uint32_t>(slab);
    if (n->bytes + slab <= max_smem) {
        n->state_in_global = false;
        n->smem = n->bytes + slab;
    } else {
        n->state_in_global = true;
        n->smem = n->bytes;
    }
    return true;
}

const csmc_net_header *header_of(const void *blob, size_t bytes) {
    if (!blob || bytes < sizeof(csmc_net_header)) return nullptr;
    const auto *h = static_cast<const csmc_net_header *>(blob);
    if (h->magic != CSMC_NET_MAGIC || h->version != CSMC_NET_VERSION || h->total_bytes > bytes) return nullptr;
    return h;
}

int ensure_buffers(csmc_net *n, uint64_t runs) {
    if (runs <= n->cap_runs) return CSMC_OK;
    cudaFree(n->d_flags);
    cudaFree(n->d_values);
    n->d_flags = nullptr;
    n->d_values = nullptr;
    n->cap_runs = 0;
    CK(cudaMalloc(&n->d_flags, runs), "cudaMalloc(flags)");
    CK(cudaMalloc(&n->d_values, runs * sizeof(double)), "cudaMalloc(values)");
    n->cap_runs = runs;
    return CSMC_OK;
}

using csmc::kReduceBlocks;
__global__ void reduce_values(const double *values, uint64_t n, double *partials) {
    csmc::reduce_block(values, n, blockIdx.x, partials + 2 * blockIdx.x);
}

int run_impl(const csmc_net *cn, const csmc_query *q, uint64_t seed, uint64_t first_run, uint64_t n_runs,
             uint8_t *flags, double *values, uint32_t *steps, uint64_t *digests, uint32_t *final_state,
             csmc_result *out, void *stream, bool verify) {
    if (!cn || !q || !out) return fail(CSMC_ERR_ARG, "null argument");
    csmc_net *n = const_cast<csmc_net *>(cn);
    if (q->kind != CSMC_QUERY_LOCATION && q->kind != CSMC_QUERY_VARIABLE) return fail(CSMC_ERR_ARG, "bad query kind");
    if (q->kind == CSMC_QUERY_VARIABLE && (q->var_id < 0 || static_cast<uint32_t>(q->var_id) >= n->h.n_vars))
        return fail(CSMC_ERR_ARG, "query variable id " + std::to_string(q->var_id) + " out of range");
    if (first_run + n_runs < first_run || first_run + n_runs > (1ull << 62))
        return fail(CSMC_ERR_ARG, "run range out of bounds");
    std::memset(out, 0, sizeof *out);
    out->runs = n_runs;
    out->lanes_per_run = n->lanes;
    out->comps_per_lane = n->comps_per_lane;
    out->runs_per_cta = n->block / n->lanes;
    out->family = n->family;
    if (n_runs == 0) return CSMC_OK;
    CK(cudaSetDevice(n->device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool need_values = q->kind == CSMC_QUERY_VARIABLE;
    if (need_values && !values) {
        int rc = ensure_buffers(n, n_runs);
        if (rc) return rc;
        values = n->d_values;
    }
    CK(cudaMemsetAsync(n->d_scratch, 0, CSMC_SCRATCH_WORDS * sizeof(unsigned long long), st), "cudaMemsetAsync");
    csmc::SimParams p{};
    p.net = csmc::layout_of(n->h);
    p.blob = n->d_blob;
    p.blob_bytes = n->bytes;
    p.state_stride = n->state_stride;
    p.loc_mode = q->kind == CSMC_QUERY_LOCATION;
    p.var_id = q->var_id;
    p.is_max = q->is_max;
    p.threshold = q->threshold;
    p.horizon = static_cast<float>(q->horizon);
    p.max_steps = q->max_steps ? q->max_steps : 10000000ull;
    p.seed = seed;
    p.first_run = first_run;
    p.n_runs = n_runs;
    p.flags = flags;
    p.values = values;
    p.steps = steps;
    p.digests = digests;
    p.final_state = final_state;
    p.scratch = n->d_scratch;
    int ctas = 0;
    p.keys = csmc::philox_keys(seed);
    for (int g = 0; g < CSMC_RACE_CLASSES; ++g) p.class_src[g] = n->class_src[g];
    int rc = n->family == 0 ? csmc::sim_max_active_ctas(n->lanes, n->comps_per_lane, verify, n->block, n->smem, &ctas)
             : n->family == 2 ? csmc::batch_max_active_ctas(verify, 0, n->block, n->smem, &ctas)
             : n->family == 4 ? csmc::coded_max_active_ctas(verify, n->slots, n->all_classed, n->block, n->smem, &ctas)
                              : csmc::serial_max_active_ctas(verify, n->slots, n->loc8, n->state_in_global, n->classes,
                                                             n->block, n->smem, &ctas);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "occupancy query");
    if (ctas < 1) return fail(CSMC_ERR_LIMIT, "kernel cannot be resident with this network (shared memory)");
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n->device), "cudaDeviceGetAttribute");
    const uint64_t runs_per_cta = static_cast<uint64_t>(n->block / n->lanes);
    uint64_t grid = static_cast<uint64_t>(sms) * static_cast<uint64_t>(ctas);
    const uint64_t needed = (n_runs + runs_per_cta - 1) / runs_per_cta;
    if (grid > needed) grid = needed;
    n->grid = static_cast<int>(grid);
    p.state_global = nullptr;
    if ((n->family == 1 || n->family == 2) && n->state_in_global) {
        const size_t need = grid * static_cast<size_t>(n->state_stride);
        if (need > n->state_bytes) {
            cudaFree(n->d_state);
            n->d_state = nullptr;
            n->state_bytes = 0;
            CK(cudaMalloc(&n->d_state, need), "cudaMalloc(run state)");
            n->state_bytes = need;
        }
        p.state_global = n->d_state;
    }
    p.state_stride = n->state_stride;
    csmc::BatchParams bp{};
    if (n->family == 2) {  // the batch kernel with a one-job table
        if (!n->d_job) CK(cudaMalloc(&n->d_job, sizeof(csmc::BatchJob)), "cudaMalloc(job table)");
        csmc::BatchJob job{};
        job.net = p.net;
        job.blob = n->d_blob;
        job.run_begin = 0;
        job.n_runs = n_runs;
        job.first_run = first_run;
        job.seed = seed;
        job.max_steps = p.max_steps;
        job.threshold = p.threshold;
        job.horizon = p.horizon;
        job.loc_mode = p.loc_mode;
        job.var_id = p.var_id;
        job.is_max = p.is_max;
        job.flags = flags;
        job.values = values;
        job.steps = steps;
        job.digests = digests;
        job.final_state = final_state;
        job.counters = n->d_scratch + 1;  // hits, steps, capped
        CK(cudaMemcpyAsync(n->d_job, &job, sizeof job, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(job table)");
        bp.jobs = n->d_job;
        bp.n_jobs = 1;
        bp.state_stride = n->state_stride;
        bp.total_runs = n_runs;
        bp.queue = n->d_scratch;
        bp.state = n->d_state;
        bp.max_vars = n->h.n_vars;
        bp.max_rate_prog = n->h.n_rate_prog;
        bp.max_comps = n->h.n_comps;
    }
    CK(cudaEventRecord(n->ev0, st), "cudaEventRecord");
    rc = n->family == 0   ? csmc::sim_launch(n->lanes, n->comps_per_lane, verify, p, static_cast<int>(grid), n->block,
                                             n->smem, st)
         : n->family == 2 ? csmc::batch_launch(verify, bp, static_cast<int>(grid), n->block, st)
         : n->family == 4 ? csmc::coded_launch(verify, n->slots, n->all_classed, p, static_cast<int>(grid), n->block,
                                               n->smem, st)
                          : csmc::serial_launch(verify, n->slots, n->loc8, n->state_in_global, n->classes, p,
                                                static_cast<int>(grid), n->block, n->smem, st);
    if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "simulation kernel launch");
    CK(cudaEventRecord(n->ev1, st), "cudaEventRecord");
    if (need_values) reduce_values<<<kReduceBlocks, 256, 0, st>>>(values, n_runs, n->d_partials);
    unsigned long long sc[CSMC_SCRATCH_WORDS];
    CK(cudaMemcpyAsync(sc, n->d_scratch, sizeof sc, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(scratch)");
    std::vector<double> part(2 * kReduceBlocks, 0.0);
    if (need_values)
        CK(cudaMemcpyAsync(part.data(), n->d_partials, part.size() * sizeof(double), cudaMemcpyDeviceToHost, st),
           "cudaMemcpyAsync(partials)");
    CK(cudaStreamSynchronize(st), "simulation kernel");
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, n->ev0, n->ev1), "cudaEventElapsedTime");
    out->kernel_ms = ms;
    out->hits = sc[1];
    out->steps = sc[2];
    out->capped = sc[3];
    for (int b = 0; b < kReduceBlocks; ++b) {
        out->sum += part[2 * b];
        out->sum_sq += part[2 * b + 1];
    }
    if (q->kind == CSMC_QUERY_VARIABLE && q->is_estimate) out->estimate = out->sum / static_cast<double>(n_runs);
    else out->estimate = static_cast<double>(out->hits) / static_cast<double>(n_runs);
    return CSMC_OK;
}

// writeTimingToCSV of the reference (simulation/write_csv.cu:15-98): one row
// per model file name, one column per "MC<n>_Sim<n>_Time<T>" configuration,
// ';'-separated, at <parent of cwd>/results5.csv.
void write_timing_csv(const std::string &xml_path, int mc, int sims, double time_bound, double ms) {
    namespace fs = std::filesystem;
    const fs::path csv = fs::current_path().parent_path() / "results5.csv";
    const std::string fname = fs::path(xml_path).filename().string();
    std::ostringstream ts;
    ts << std::fixed << std::setprecision(2) << time_bound;
    const std::string config = "MC" + std::to_string(mc) + "_Sim" + std::to_string(sims) + "_Time" + ts.str();
    std::vector<std::vector<std::string>> rows;
    if (fs::exists(csv)) {
        std::ifstream f(csv);
        std::string line;
        while (std::getline(f, line)) {
            std::vector<std::string> row;
            std::stringstream ls(line);
            std::string cell;
            while (std::getline(ls, cell, ';')) row.push_back(cell);
            rows.push_back(row);
        }
    }
    if (rows.empty()) rows.push_back({""});
    size_t col = 0;
    for (size_t c = 1; c < rows[0].size(); ++c)
        if (rows[0][c] == config) { col = c; break; }
    if (!col) {
        col = rows[0].size();
        rows[0].push_back(config);
    }
    size_t row = 0;
    for (size_t r = 1; r < rows.size(); ++r)
        if (!rows[r].empty() && rows[r][0] == fname) { row = r; break; }
    if (!row) {
        row = rows.size();
        rows.push_back({fname});
    }
    for (auto &r : rows)
        while (r.size() <= col) r.push_back("");
    rows[row][col] = std::to_string(ms);
    std::ofstream o(csv);
    if (!o.is_open()) {
        std::cerr << "Failed to open file for writing" << std::endl;
        return;
    }
    for (const auto &r : rows) {
        o << r[0];
        for (size_t i = 1; i < r.size(); ++i) o << ";" << r[i];
        o << "\n";
    }
}

}  // namespace

namespace csmc {
// Lets other translation units of the library report through csmc_last_error().
void set_last_error(const std::string &m) { g_err = m; }
}  // namespace csmc

extern "C" {

const char *csmc_last_error(void) { return g_err.c_str(); }

const char *csmc_version(void) { return "csmc-b200 0.1 (sm_100a)"; }

void csmc_free(void *p) { std::free(p); }

int csmc_model_compile(const char *xml_path, const char *loc_query, int loc_mode, void **blob, size_t *bytes) {
    if (!xml_path || !blob || !bytes) return fail(CSMC_ERR_ARG, "null argument");
    try {
        auto net = csmc::parse_uppaal_file(xml_path);
        csmc::DevModel m = csmc::build_device_model(*net, loc_query ? loc_query : "", loc_mode != 0);
        std::vector<uint8_t> b = csmc::pack_device_model(m);
        void *p = std::malloc(b.size());
        if (!p) return fail(CSMC_ERR_ARG, "out of host memory");
        std::memcpy(p, b.data(), b.size());
        *blob = p;
        *bytes = b.size();
        return CSMC_OK;
    } catch (const std::exception &e) {
        return fail(CSMC_ERR_MODEL, e.what());
    }
}

int csmc_model_dump(const char *xml_path, const char *loc_query, int loc_mode, char **text) {
    if (!xml_path || !text) return fail(CSMC_ERR_ARG, "null argument");
    try {
        auto net = csmc::parse_uppaal_file(xml_path);
        csmc::DevModel m = csmc::build_device_model(*net, loc_query ? loc_query : "", loc_mode != 0);
        const std::string s = csmc::dump_device_model(m);
        char *p = static_cast<char *>(std::malloc(s.size() + 1));
        std::memcpy(p, s.c_str(), s.size() + 1);
        *text = p;
        return CSMC_OK;
    } catch (const std::exception &e) {
        return fail(CSMC_ERR_MODEL, e.what());
    }
}

int csmc_blob_info(const void *blob, size_t bytes, uint32_t *n_vars, uint32_t *n_comps, uint32_t *n_locs) {
    const csmc_net_header *h = header_of(blob, bytes);
    if (!h) return fail(CSMC_ERR_ARG, "not a network blob");
    if (n_vars) *n_vars = h->n_vars;
    if (n_comps) *n_comps = h->n_comps;
    if (n_locs) *n_locs = h->n_locs;
    return CSMC_OK;
}

int csmc_net_upload(const void *blob, size_t bytes, csmc_net **out) {
    if (!out) return fail(CSMC_ERR_ARG, "null argument");
    *out = nullptr;
    const csmc_net_header *h = header_of(blob, bytes);
    if (!h) return fail(CSMC_ERR_ARG, "not a network blob");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(CSMC_ERR_NODEVICE, "no CUDA device is available (there is no CPU fallback)");
    }
    auto n = std::make_unique<csmc_net>();
    CK(cudaGetDevice(&n->device), "cudaGetDevice");
    n->h = *h;
    n->bytes = (h->total_bytes + 15u) & ~15u;
    n->slots = h->max_edges_per_loc >= 2;
    n->loc8 = h->max_locs_per_comp <= 256;
    n->classes = (h->flags & CSMC_NET_RACE_CLASSES) != 0 && h->n_comps <= 256;
    if (n->classes && h->off_loc_desc + 8ull * h->n_locs > h->total_bytes)
        return fail(CSMC_ERR_ARG, "not a network blob (descriptor table out of range)");
    if (n->classes) {
        // each class's 1/rate source, and whether every location is classed
        // (the class-coded kernel's launch parameters)
        const uint8_t *base = static_cast<const uint8_t *>(blob);
        n->all_classed = true;
        for (uint32_t i = 0; i < h->n_locs; ++i) {
            uint64_t d;
            std::memcpy(&d, base + h->off_loc_desc + 8ull * i, 8);
            const uint32_t lo = static_cast<uint32_t>(d), fl = static_cast<uint32_t>(d >> 32);
            const uint32_t g = CSMC_DESC_CLASS(fl);
            if (g >= CSMC_RACE_CLASSES) {
                n->all_classed = false;
                continue;
            }
            n->class_src[g] = (fl & CSMC_DESC_PROG) ? (CSMC_CLASS_SRC_PROG | lo) : lo;
        }
        // tilt groups of importance sampling one thread per run: the
        // (race class, location class) pairs in order of first appearance,
        // the first CSMC_IS_GROUPS of them; later pairs take the
        // descriptor path (code 7)
        if (h->n_comps >= 4 && h->max_locs_per_comp <= 32 && h->off_comp + 8ull * h->n_comps <= h->total_bytes) {
            int8_t id[CSMC_RACE_CLASSES][4];
            std::memset(id, -1, sizeof id);
            int groups = 0;
            uint64_t map = 0;
            for (uint32_t c = 0; c < h->n_comps; ++c) {
                csmc_comp cp;
                std::memcpy(&cp, base + h->off_comp + 8ull * c, sizeof cp);
                for (uint32_t k = 0; k < cp.n_locs && cp.loc_begin + k < h->n_locs; ++k) {
                    uint64_t d;
                    std::memcpy(&d, base + h->off_loc_desc + 8ull * (cp.loc_begin + k), 8);
                    const uint32_t g = CSMC_DESC_CLASS(static_cast<uint32_t>(d >> 32));
                    if (g >= CSMC_RACE_CLASSES || id[g][k & 3u] >= 0) continue;
                    id[g][k & 3u] = static_cast<int8_t>(groups < CSMC_IS_GROUPS ? groups : 7);
                    if (groups < CSMC_IS_GROUPS) {
                        n->is_group_src[groups] = n->class_src[g];
                        n->is_group_l |= (k & 3u) << (2 * groups);
                        ++groups;
                    }
                }
            }
            for (uint32_t g = 0; g < CSMC_RACE_CLASSES; ++g)
                for (uint32_t l = 0; l < 4; ++l)
                    map |= static_cast<uint64_t>(id[g][l] < 0 ? 7 : id[g][l]) << (3 * (4 * g + l));
            n->is_group_map = map;
            n->is_groups = groups;
            bool spill = false;  // a classed location's pair beyond the groups
            for (uint32_t g = 0; g < CSMC_RACE_CLASSES; ++g)
                for (uint32_t l = 0; l < 4; ++l) spill = spill || id[g][l] == 7;
            n->is_all_grouped = n->all_classed && !spill && h->n_comps % 4 == 0;
        }
    }
    // default plan: the class-coded thread-per-run kernel when the network
    // has race classes and fits its limits; else one thread per run when the
    // run state of a 128-thread CTA fits next to the network in shared
    // memory, lane groups otherwise
    std::string why;
    int G = 0, K = 0;
    choose_shape(h->n_comps, G, K);
    const size_t per_thread = csmc::serial_state_bytes_per_thread(h->n_comps, h->n_vars, h->n_rate_prog, n->slots, n->loc8);
    const bool serial_fits = n->bytes + 128 * per_thread <= static_cast<size_t>(max_smem_optin(n->device));
    bool ok = configure_plan(n.get(), 4, 1, static_cast<int>(h->n_comps), 128, why);
    if (!ok && serial_fits) ok = configure_plan(n.get(), 1, 1, static_cast<int>(h->n_comps), 128, why);
    if (!ok) ok = configure_plan(n.get(), 0, G, K, 256, why);
    if (!ok) ok = configure_plan(n.get(), 1, 1, static_cast<int>(h->n_comps), 128, why);
    if (!ok) ok = configure_plan(n.get(), 2, 1, static_cast<int>(h->n_comps), 128, why);
    if (!ok) return fail(CSMC_ERR_LIMIT, "no launch plan for this network: " + why);
    CK(cudaMalloc(&n->d_blob, n->bytes), "cudaMalloc(network)");
    CK(cudaMemset(n->d_blob, 0, n->bytes), "cudaMemset");
    CK(cudaMemcpy(n->d_blob, blob, h->total_bytes, cudaMemcpyHostToDevice), "cudaMemcpy(network)");
    CK(cudaMalloc(&n->d_scratch, CSMC_SCRATCH_WORDS * sizeof(unsigned long long)), "cudaMalloc(scratch)");
    CK(cudaMalloc(&n->d_partials, 2 * kReduceBlocks * sizeof(double)), "cudaMalloc(partials)");
    CK(cudaEventCreate(&n->ev0), "cudaEventCreate");
    CK(cudaEventCreate(&n->ev1), "cudaEventCreate");
    *out = n.release();
    return CSMC_OK;
}

void csmc_net_free(csmc_net *n) {
    if (!n) return;
    cudaFree(n->d_blob);
    cudaFree(n->d_scratch);
    cudaFree(n->d_flags);
    cudaFree(n->d_values);
    cudaFree(n->d_partials);
    cudaFree(n->d_state);
    cudaFree(n->d_job);
    cudaFree(n->d_mlp);
    cudaFree(n->d_wvals);
    cudaFree(n->d_is_flags);
    cudaFree(n->d_theta_cache);
    if (n->ev0) cudaEventDestroy(n->ev0);
    if (n->ev1) cudaEventDestroy(n->ev1);
    delete n;
}

int csmc_set_plan(csmc_net *n, int32_t family, int32_t lanes_per_run, int32_t comps_per_lane,
                  int32_t threads_per_cta) {
    if (!n) return fail(CSMC_ERR_ARG, "null argument");
    const csmc_net saved = *n;
    std::string why;
    if (!configure_plan(n, family, lanes_per_run, comps_per_lane, threads_per_cta, why)) {
        n->family = saved.family;
        n->lanes = saved.lanes;
        n->comps_per_lane = saved.comps_per_lane;
        n->block = saved.block;
        n->smem = saved.smem;
        n->state_stride = saved.state_stride;
        n->state_in_global = saved.state_in_global;
        return fail(CSMC_ERR_ARG, "plan rejected: " + why);
    }
    return CSMC_OK;
}

int csmc_plan(const csmc_net *n, int32_t *lanes, int32_t *cpl, int32_t *rpc) {
    if (!n) return fail(CSMC_ERR_ARG, "null argument");
    if (lanes) *lanes = n->lanes;
    if (cpl) *cpl = n->comps_per_lane;
    if (rpc) *rpc = n->block / n->lanes;
    return CSMC_OK;
}

int csmc_run(const csmc_net *net, const csmc_query *q, uint64_t seed, uint64_t first_run, uint64_t n_runs,
             uint8_t *flags, double *values, uint32_t *steps, csmc_result *out, void *stream) {
    try {
        return run_impl(net, q, seed, first_run, n_runs, flags, values, steps, nullptr, nullptr, out, stream, false);
    } catch (const std::exception &e) {
        return fail(CSMC_ERR_ARG, e.what());
    }
}

int csmc_run_verify(const csmc_net *net, const csmc_query *q, uint64_t seed, uint64_t first_run, uint64_t n_runs,
                    uint8_t *flags, double *values, uint32_t *steps, uint64_t *digests, uint32_t *final_state,
                    csmc_result *out, void *stream) {
    try {
        return run_impl(net, q, seed, first_run, n_runs, flags, values, steps, digests, final_state, out, stream,
                        true);
    } catch (const std::exception &e) {
        return fail(CSMC_ERR_ARG, e.what());
    }
}

}  // extern "C"

namespace {

std::string json_escape(const std::string &s) {
    std::string o;
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o;
}

// The reference's smc() flow (smc.cu:283-491) for one query, plus the
// optional JSON summary and per-run dump of csmc_smc_ex.
int smc_impl(const char *model_path, int seed, int sims, const csmc_query &q0, const std::string &lq,
             const char *json_path, const char *runs_path) {
    if (!model_path) return fail(CSMC_ERR_ARG, "null model path");
    const bool loc_mode = q0.kind == CSMC_QUERY_LOCATION;
    void *blob = nullptr;
    size_t bytes = 0;
    int rc = csmc_model_compile(model_path, lq.c_str(), loc_mode ? 1 : 0, &blob, &bytes);
    if (rc) return rc;
    const csmc_net_header *h = header_of(blob, bytes);
    std::printf("Set number of variables to: %d\n", static_cast<int>(h->n_vars));
    std::fflush(stdout);
    const int mc = static_cast<int>(h->n_comps);
    const double time_bound = q0.horizon;
    std::cout << "=================\n\n";
    std::cout << "Running SMC with the following settings:" << std::endl;
    std::cout << "- Number of simulations: " << sims << std::endl;
    std::cout << "- Model: " << model_path << std::endl;
    std::cout << "- Random seed: " << seed << std::endl;
    std::cout << "- Time bound: " << time_bound << std::endl;
    std::cout << "- Num components: " << mc << std::endl;
    if (!loc_mode)
        std::cout << "- Logging type: variable query. Finding " << (q0.is_max ? "max" : "min")
                  << " of variable with ID " << q0.var_id << std::endl;
    else
        std::cout << "- Logging type: location query on query: " << lq << std::endl;
    std::cout << "=================\n\n";

    csmc_query q = q0;
    q.horizon = static_cast<double>(static_cast<float>(time_bound));
    const uint64_t n_runs = sims > 0 ? static_cast<uint64_t>(sims) : 0;
    std::vector<uint8_t> flags(n_runs);
    std::vector<double> values(n_runs);
    csmc_result res{};
    const auto t0 = std::chrono::steady_clock::now();
    rc = csmc_run_host(blob, bytes, &q, static_cast<uint64_t>(static_cast<int64_t>(seed)), 0, n_runs, flags.data(),
                       values.data(), nullptr, &res);
    const auto dur = std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0);
    std::free(blob);
    if (rc) {
        std::cout << "Error: " << g_err << std::endl;
        return rc;
    }
    const double ms = dur.count() / 1000000.0;
    std::cout << "Time taken: " << ms << " ms on file " << model_path << std::endl;
    std::cout << "Time taken: " << dur.count() << " on file " << model_path << std::endl;
    std::cout << "Time taken: " << dur.count() << " ns (" << (dur.count() / 1000000.0) << " ms)" << std::endl;
    write_timing_csv(model_path, mc, sims, time_bound, ms);
    double result = 0, sum_sq = 0;
    uint64_t hits = 0;
    if (!loc_mode) {
        if (q.is_estimate) {
            for (uint64_t i = 0; i < n_runs; ++i) {
                result += values[i];
                sum_sq += values[i] * values[i];
            }
            result = result / static_cast<double>(sims);
        } else {
            for (uint64_t i = 0; i < n_runs; ++i) {
                if (q.is_max && values[i] > q.threshold) ++hits;
                if (!q.is_max && values[i] < q.threshold) ++hits;
            }
            result = static_cast<double>(hits) / static_cast<double>(sims);
        }
        std::cout << "Result: " << result << std::endl;
    } else {
        for (uint64_t i = 0; i < n_runs; ++i)
            if (flags[i]) ++hits;
        std::cout << "Number of simulations: " << n_runs << std::endl;
        std::cout << "Number of hits: " << hits << std::endl;
        std::cout << "The answer to " << lq << " is "
                  << static_cast<float>(hits) / static_cast<float>(sims) << std::endl;
        result = static_cast<double>(hits) / static_cast<double>(sims);
    }
    if (runs_path && *runs_path) {
        std::ofstream o(runs_path);
        if (!o) return fail(CSMC_ERR_ARG, std::string("cannot write ") + runs_path);
        o << "run,flag,value\n";
        o << std::setprecision(17);
        for (uint64_t i = 0; i < n_runs; ++i) o << i << ',' << static_cast<int>(flags[i]) << ',' << values[i] << '\n';
    }
    if (json_path && *json_path) {
        const double n = static_cast<double>(n_runs);
        const bool estimate = !loc_mode && q.is_estimate;
        double half = 0.0;
        if (n_runs > 0) {
            if (estimate) {
                const double var = n > 1 ? std::max(0.0, (sum_sq - n * result * result) / (n - 1)) : 0.0;
                half = 1.96 * std::sqrt(var / n);
            } else {
                half = 1.96 * std::sqrt(std::max(0.0, result * (1 - result)) / n);
            }
        }
        const double delta = 0.05;
        const double eps = n_runs ? std::sqrt(std::log(2 / delta) / (2 * n)) : 0.0;
        std::ofstream o(json_path);
        if (!o) return fail(CSMC_ERR_ARG, std::string("cannot write ") + json_path);
        o << std::setprecision(17);
        o << "{\"model\": \"" << json_escape(model_path) << "\", \"seed\": " << seed << ", \"simulations\": " << n_runs
          << ", \"query\": {\"kind\": \"" << (loc_mode ? "location" : "variable") << "\", \"var_id\": " << q.var_id
          << ", \"is_max\": " << q.is_max << ", \"is_estimate\": " << q.is_estimate << ", \"threshold\": " << q.threshold
          << ", \"time_bound\": " << time_bound << ", \"location\": \"" << json_escape(lq) << "\"}"
          << ", \"result\": " << result << ", \"hits\": " << hits << ", \"ci95\": [" << result - half << ", "
          << result + half << "]"
          << ", \"chernoff_hoeffding\": {\"delta\": " << delta << ", \"epsilon\": " << eps
          << ", \"runs_for_epsilon_0_01\": " << std::ceil(std::log(2 / delta) / (2 * 0.01 * 0.01)) << "}"
          << ", \"race_steps\": " << res.steps << ", \"capped_runs\": " << res.capped << ", \"ms\": " << ms << "}\n";
    }
    return CSMC_OK;
}

}  // namespace

extern "C" {

int csmc_smc(const char *model_path, int seed, int sims, int time_bound, int threshold, int var_id, int is_max,
             int is_estimate, const char *loc_query) {
    csmc_query q{};
    q.kind = var_id == -1 ? CSMC_QUERY_LOCATION : CSMC_QUERY_VARIABLE;
    q.var_id = var_id;
    q.is_max = is_max;
    q.is_estimate = is_estimate;
    q.threshold = threshold;
    q.horizon = time_bound;
    return smc_impl(model_path, seed, sims, q, loc_query ? loc_query : "", nullptr, nullptr);
}

int csmc_smc_ex(const char *model_path, int seed, int sims, const csmc_query *q, const char *loc_query,
                const char *json_path, const char *runs_path) {
    if (!q) return fail(CSMC_ERR_ARG, "null query");
    return smc_impl(model_path, seed, sims, *q, loc_query ? loc_query : "", json_path, runs_path);
}

int csmc_query_parse(const char *xml_path, const char *formula, csmc_query *q, char *loc_query, size_t loc_cap,
                     uint64_t *sims) {
    if (!xml_path || !formula || !q) return fail(CSMC_ERR_ARG, "null argument");
    std::unique_ptr<csmc::Network> net;
    try {
        net = csmc::parse_uppaal_file(xml_path);
    } catch (const std::exception &e) {
        return fail(CSMC_ERR_MODEL, e.what());
    }
    try {
        const csmc::QueryText t = csmc::parse_formula(*net, formula);
        std::memset(q, 0, sizeof *q);
        q->kind = t.kind == 0 ? CSMC_QUERY_LOCATION : CSMC_QUERY_VARIABLE;
        q->var_id = t.var_id;
        q->is_max = t.is_max;
        q->is_estimate = t.is_estimate;
        q->threshold = t.threshold;
        q->horizon = t.horizon;
        if (loc_query) {
            if (t.loc_query.size() + 1 > loc_cap) return fail(CSMC_ERR_ARG, "location buffer too small");
            std::memcpy(loc_query, t.loc_query.c_str(), t.loc_query.size() + 1);
        }
        if (sims) *sims = t.sims;
        return CSMC_OK;
    } catch (const std::exception &e) {
        return fail(CSMC_ERR_ARG, e.what());
    }
}

}  // extern "C"
