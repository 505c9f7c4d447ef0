// csmc_run_noalloc: the thread-per-run simulation without any device memory
// allocation by this library.
//
// Who needs it: hosts that own every byte of device memory themselves and do
// not let plug-ins call cudaMalloc/cudaFree — a process that reserves a fixed
// pool at start-up and runs with allocation disabled afterwards, a latency-
// critical loop in which cudaMalloc's implicit device synchronisation is not
// acceptable, or an embedding framework whose allocator is the only one
// allowed to touch the device.  Such a caller places the packed network,
// the per-run output buffers and nothing else; the scratch memory the kernel
// needs (work counter, hit/step counters, the partial sums of the values,
// and per-CTA run-state slabs for networks whose run state does not fit in
// shared memory) comes from the file-scope array below, which every GPU that
// loads the library holds for as long as the process lives.
#include "../../include/csmc.h"
#include "include/csmc_net.h"
#include "include/csmc_numeric.h"
#include "kernels/reduce.cuh"
#include "kernels/sim.cuh"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

namespace csmc {
void set_last_error(const std::string &m);  // capi.cu
}

namespace {

// Scratch of the no-allocation entry point: CSMC_NOALLOC_SCRATCH_BYTES
// bytes per device.  Layout: [0, 64) counters, [64, 64 + 4096) partial sums,
// [kSlabOffset, end) run-state slabs of the thread-per-run kernel.
constexpr size_t kScratchBytes = CSMC_NOALLOC_SCRATCH_BYTES;
using csmc::kReduceBlocks;
constexpr size_t kPartialOffset = 64;
constexpr size_t kSlabOffset = 8192;
static_assert(kPartialOffset + 2 * kReduceBlocks * sizeof(double) <= kSlabOffset, "scratch layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

int fail(int code, const std::string &m) {
    csmc::set_last_error(m);  // reported by csmc_last_error()
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(CSMC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// The current context's unique id (cuCtxGetId), through driver entry points
// fetched from the runtime, so the library does not link the driver itself.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

int current_context_id(int dev, unsigned long long *id) {
    static std::once_flag once;
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    std::call_once(once, [] {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa{}, qb{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(a);
        if (cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(b);
        cudaGetLastError();
    });
    if (!get_current || !get_id) return fail(CSMC_ERR_CUDA, "driver entry points cuCtxGetCurrent/cuCtxGetId");
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) {
        // no context current on this thread yet: make the device's primary
        // context current (cudaSetDevice initialises it)
        const cudaError_t e = cudaSetDevice(dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
        if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return fail(CSMC_ERR_CUDA, "no current CUDA context");
    }
    if (get_id(ctx, id) != CUDA_SUCCESS) return fail(CSMC_ERR_CUDA, "cuCtxGetId");
    return CSMC_OK;
}

// Device address of g_noalloc_scratch per device ordinal, looked up with
// that device current and kept together with the id of the context it was
// looked up in: a call from another context on the same device (after a
// cudaDeviceReset, or from a non-primary context) looks the address up
// again instead of using a stale one.  In host code the symbol itself is
// only a host-side stand-in, never a device address.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

int scratch_for_current_device(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(CSMC_ERR_LIMIT, "device ordinal out of range");
    unsigned long long ctx = 0;
    int rc = current_context_id(dev, &ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_scratch_ptr[dev] = p;
        g_scratch_ctx[dev] = ctx;
    }
    *out = g_scratch_ptr[dev];
    return CSMC_OK;
}

// Deterministic sum and sum of squares of values[0..n) into partials[2*b],
// partials[2*b+1] per block b: csmc_run's reduction (kernels/reduce.cuh),
// so the sums carry the same bits as csmc_run's.
__global__ void noalloc_reduce(const double *values, uint64_t n, double *partials) {
    csmc::reduce_block(values, n, blockIdx.x, partials + 2 * blockIdx.x);
}

}  // namespace

extern "C" int csmc_run_noalloc(const void *blob_host, const void *blob_device, size_t bytes, const csmc_query *q,
                                uint64_t seed, uint64_t first_run, uint64_t n_runs, uint8_t *flags, double *values,
                                uint32_t *steps, csmc_result *out, void *stream) {
    try {
        if (!blob_host || !blob_device || !q || !out) return fail(CSMC_ERR_ARG, "null argument");
        if (bytes < sizeof(csmc_net_header)) return fail(CSMC_ERR_ARG, "blob too small");
        csmc_net_header h;
        std::memcpy(&h, blob_host, sizeof h);
        if (h.magic != CSMC_NET_MAGIC || h.version != CSMC_NET_VERSION || h.total_bytes > bytes ||
            h.total_bytes % 16)
            return fail(CSMC_ERR_ARG, "not a network blob");
        if (reinterpret_cast<uintptr_t>(blob_device) % 16) return fail(CSMC_ERR_ARG, "device blob must be 16-byte aligned");
        if (q->kind != CSMC_QUERY_LOCATION && q->kind != CSMC_QUERY_VARIABLE) return fail(CSMC_ERR_ARG, "bad query kind");
        if (q->kind == CSMC_QUERY_VARIABLE && (q->var_id < 0 || static_cast<uint32_t>(q->var_id) >= h.n_vars))
            return fail(CSMC_ERR_ARG, "query variable id out of range");
        if (q->kind == CSMC_QUERY_VARIABLE && !values)
            return fail(CSMC_ERR_ARG, "variable queries need a values buffer (nothing is allocated here)");
        if (first_run + n_runs < first_run || first_run + n_runs > (1ull << 62))
            return fail(CSMC_ERR_ARG, "run range out of bounds");
        std::memset(out, 0, sizeof *out);
        out->runs = n_runs;
        if (n_runs == 0) return CSMC_OK;

        void *scratch = nullptr;
        int rc = scratch_for_current_device(&scratch);
        if (rc) return rc;
        int dev = 0, sms = 0, max_smem = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e != cudaSuccess) return cuda_fail(e, "device attributes");

        // plan: one thread per run, 128 threads per CTA; run state in shared
        // memory when it fits, otherwise in slabs of the scratch array
        const bool slots = h.max_edges_per_loc >= 2;
        const bool loc8 = h.max_locs_per_comp <= 256;
        const bool classes = (h.flags & CSMC_NET_RACE_CLASSES) != 0 && h.n_comps <= 256;
        const uint32_t blob_bytes = h.total_bytes;
        if (blob_bytes > static_cast<uint32_t>(max_smem))
            return fail(CSMC_ERR_LIMIT, "network does not fit in shared memory");
        const int block = 128;
        const size_t per_thread = csmc::serial_state_bytes_per_thread(h.n_comps, h.n_vars, h.n_rate_prog, slots, loc8);
        const size_t slab = (per_thread * block + 15) & ~static_cast<size_t>(15);
        const bool in_smem = blob_bytes + slab <= static_cast<size_t>(max_smem);
        const size_t smem = in_smem ? blob_bytes + slab : blob_bytes;
        int ctas = 0;
        rc = csmc::serial_max_active_ctas(false, slots, loc8, !in_smem, classes, block, smem, &ctas);
        if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "occupancy query");
        if (ctas < 1) return fail(CSMC_ERR_LIMIT, "kernel cannot be resident with this network");
        uint64_t grid = static_cast<uint64_t>(sms) * static_cast<uint64_t>(ctas);
        const uint64_t needed = (n_runs + block - 1) / block;
        if (grid > needed) grid = needed;
        uint8_t *base = static_cast<uint8_t *>(scratch);
        if (!in_smem) {
            const uint64_t fit = (kScratchBytes - kSlabOffset) / slab;
            if (fit < 1)
                return fail(CSMC_ERR_LIMIT, "run state of this network needs " + std::to_string(slab) +
                                                " bytes per CTA; the no-allocation entry point has " +
                                                std::to_string(kScratchBytes - kSlabOffset) + " bytes of scratch");
            if (grid > fit) grid = fit;
        }

        cudaStream_t st = static_cast<cudaStream_t>(stream);
        e = cudaMemsetAsync(base, 0, kPartialOffset, st);  // counters start at zero
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(scratch)");
        csmc::SimParams p{};
        p.net = csmc::layout_of(h);
        p.blob = static_cast<const uint8_t *>(blob_device);
        p.blob_bytes = blob_bytes;
        p.state_stride = static_cast<uint32_t>(slab);
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
        p.scratch = reinterpret_cast<unsigned long long *>(base);
        p.state_global = in_smem ? nullptr : base + kSlabOffset;
        rc = csmc::serial_launch(false, slots, loc8, !in_smem, classes, p, static_cast<int>(grid), block, smem, st);
        if (rc) return cuda_fail(static_cast<cudaError_t>(rc), "simulation kernel launch");
        double *partials = reinterpret_cast<double *>(base + kPartialOffset);
        const bool need_values = q->kind == CSMC_QUERY_VARIABLE;
        if (need_values) noalloc_reduce<<<kReduceBlocks, 256, 0, st>>>(values, n_runs, partials);
        unsigned long long sc[CSMC_SCRATCH_WORDS];
        e = cudaMemcpyAsync(sc, base, sizeof sc, cudaMemcpyDeviceToHost, st);
        double part[2 * kReduceBlocks] = {};
        if (e == cudaSuccess && need_values)
            e = cudaMemcpyAsync(part, partials, sizeof part, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "simulation kernel");
        out->hits = sc[1];
        out->steps = sc[2];
        out->capped = sc[3];
        for (int b = 0; b < kReduceBlocks; ++b) {
            out->sum += part[2 * b];
            out->sum_sq += part[2 * b + 1];
        }
        if (q->kind == CSMC_QUERY_VARIABLE && q->is_estimate) out->estimate = out->sum / static_cast<double>(n_runs);
        else out->estimate = static_cast<double>(out->hits) / static_cast<double>(n_runs);
        out->lanes_per_run = 1;
        out->comps_per_lane = static_cast<int32_t>(h.n_comps);
        out->runs_per_cta = block;
        out->family = 1;
        return CSMC_OK;
    } catch (const std::exception &ex) {
        return fail(CSMC_ERR_ARG, ex.what());
    }
}
