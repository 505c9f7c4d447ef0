// csmc_run_host: the simulation from a host network blob to host outputs,
// the call a host program (the CLI, smc()) makes per query.
//
// Per device the library keeps one host-path context: the network handle of
// the last blob (its upload and launch plan), device output buffers, a
// pinned copy of the blob and pinned staging buffers, and a stream.  A call
// with the same blob bytes as the previous one on that device reuses the
// plan and the buffers; the blob itself is still copied to the device on
// every call (the step's input crosses the bus every time).  Results come
// back through the pinned staging buffers in chunks: the copy of chunk k+1
// runs while chunk k is copied into the caller's buffers and summed, in run
// order, as the reference's host reduction does (smc.cu:378-402).
//
// Calls on one device are serialised by a mutex; the context's memory is
// held until csmc_run_host_release() or process exit.
#include "../../include/csmc.h"
#include "capi_internal.h"

#include <cuda_runtime.h>

#include <cstring>
#include <memory>
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

#define HCK(x, what)                                       \
    do {                                                   \
        cudaError_t e_ = (x);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

constexpr size_t kChunkBytes = 4u << 20;  // one pinned staging chunk

struct HostPath {
    std::mutex mu;
    std::vector<uint8_t> blob;  // bytes of the network behind `net`
    csmc_net *net = nullptr;
    uint8_t *h_blob = nullptr;  // pinned copy of the blob for the upload
    size_t h_blob_cap = 0;
    uint8_t *d_flags = nullptr;
    double *d_values = nullptr;
    uint32_t *d_steps = nullptr;
    uint64_t cap = 0, steps_cap = 0;
    uint8_t *stage[2] = {nullptr, nullptr};  // pinned, kChunkBytes each
    cudaStream_t stream = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};

    void release() {
        if (net) csmc_net_free(net);
        net = nullptr;
        blob.clear();
        cudaFreeHost(h_blob);
        h_blob = nullptr;
        h_blob_cap = 0;
        cudaFree(d_flags);
        cudaFree(d_values);
        cudaFree(d_steps);
        d_flags = nullptr;
        d_values = nullptr;
        d_steps = nullptr;
        cap = steps_cap = 0;
        for (int i = 0; i < 2; ++i) {
            cudaFreeHost(stage[i]);
            stage[i] = nullptr;
            if (done[i]) cudaEventDestroy(done[i]);
            done[i] = nullptr;
        }
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }
};

constexpr int kMaxDevices = 64;
std::mutex g_paths_mu;
HostPath *g_paths[kMaxDevices] = {};  // never destroyed: process exit tears the CUDA context down

HostPath *path_of(int dev) {
    std::lock_guard<std::mutex> lock(g_paths_mu);
    if (!g_paths[dev]) g_paths[dev] = new HostPath();
    return g_paths[dev];
}

int prepare(HostPath &hp, const void *blob, size_t bytes, uint64_t n_runs, bool want_steps) {
    if (!hp.stream) HCK(cudaStreamCreateWithFlags(&hp.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (int i = 0; i < 2; ++i) {
        if (!hp.stage[i]) HCK(cudaMallocHost(&hp.stage[i], kChunkBytes), "cudaMallocHost(staging)");
        if (!hp.done[i]) HCK(cudaEventCreateWithFlags(&hp.done[i], cudaEventDisableTiming), "cudaEventCreate");
    }
    // the network: reuse the handle (upload, plan) when the bytes are the same
    const bool same = hp.net && hp.blob.size() == bytes && std::memcmp(hp.blob.data(), blob, bytes) == 0;
    if (!same) {
        if (hp.net) csmc_net_free(hp.net);
        hp.net = nullptr;
        hp.blob.clear();
        int rc = csmc_net_upload(blob, bytes, &hp.net);
        if (rc) return rc;
        hp.blob.assign(static_cast<const uint8_t *>(blob), static_cast<const uint8_t *>(blob) + bytes);
    }
    // this call's input crosses to the device: blob -> pinned -> network buffer
    if (hp.h_blob_cap < bytes) {
        cudaFreeHost(hp.h_blob);
        hp.h_blob = nullptr;
        hp.h_blob_cap = 0;
        HCK(cudaMallocHost(&hp.h_blob, bytes), "cudaMallocHost(network)");
        hp.h_blob_cap = bytes;
    }
    std::memcpy(hp.h_blob, blob, bytes);
    HCK(cudaMemcpyAsync(hp.net->d_blob, hp.h_blob, hp.net->h.total_bytes, cudaMemcpyHostToDevice, hp.stream),
        "cudaMemcpyAsync(network)");
    // device outputs, grown geometrically
    if (n_runs > hp.cap) {
        const uint64_t c = n_runs + n_runs / 2;
        cudaFree(hp.d_flags);
        cudaFree(hp.d_values);
        hp.d_flags = nullptr;
        hp.d_values = nullptr;
        hp.cap = 0;
        HCK(cudaMalloc(&hp.d_flags, c), "cudaMalloc(flags)");
        HCK(cudaMalloc(&hp.d_values, c * sizeof(double)), "cudaMalloc(values)");
        hp.cap = c;
    }
    if (want_steps && n_runs > hp.steps_cap) {
        const uint64_t c = n_runs + n_runs / 2;
        cudaFree(hp.d_steps);
        hp.d_steps = nullptr;
        hp.steps_cap = 0;
        HCK(cudaMalloc(&hp.d_steps, c * sizeof(uint32_t)), "cudaMalloc(steps)");
        hp.steps_cap = c;
    }
    return CSMC_OK;
}

// Copies n elements of `elem` bytes from device src to host dst (may be
// NULL: nothing kept) through the two pinned chunks; `each(chunk, count,
// first)` sees every chunk in order while the next one is in flight.
template <class F>
int copy_back(HostPath &hp, const void *src, size_t elem, uint64_t n, void *dst, F each) {
    const uint64_t per = kChunkBytes / elem;
    const uint64_t chunks = (n + per - 1) / per;
    auto issue = [&](uint64_t k) -> cudaError_t {
        const uint64_t first = k * per, cnt = (first + per < n) ? per : n - first;
        cudaError_t e = cudaMemcpyAsync(hp.stage[k & 1], static_cast<const uint8_t *>(src) + first * elem,
                                        cnt * elem, cudaMemcpyDeviceToHost, hp.stream);
        if (e == cudaSuccess) e = cudaEventRecord(hp.done[k & 1], hp.stream);
        return e;
    };
    if (chunks) HCK(issue(0), "cudaMemcpyAsync(results)");
    for (uint64_t k = 0; k < chunks; ++k) {
        if (k + 1 < chunks) HCK(issue(k + 1), "cudaMemcpyAsync(results)");
        HCK(cudaEventSynchronize(hp.done[k & 1]), "result copy");
        const uint64_t first = k * per, cnt = (first + per < n) ? per : n - first;
        if (dst) std::memcpy(static_cast<uint8_t *>(dst) + first * elem, hp.stage[k & 1], cnt * elem);
        each(hp.stage[k & 1], cnt, first);
    }
    return CSMC_OK;
}

int run_host(const void *blob, size_t bytes, const csmc_query *q, uint64_t seed, uint64_t first_run,
             uint64_t n_runs, uint8_t *flags, double *values, uint32_t *steps, csmc_result *out) {
    if (!blob || !q || !out) return fail(CSMC_ERR_ARG, "null argument");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(CSMC_ERR_NODEVICE, "no CUDA device is available (there is no CPU fallback)");
    }
    int dev = 0;
    HCK(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(CSMC_ERR_LIMIT, "device ordinal out of range");
    HostPath &hp = *path_of(dev);
    std::lock_guard<std::mutex> lock(hp.mu);
    int rc = prepare(hp, blob, bytes, n_runs, steps != nullptr);
    if (rc) return rc;
    rc = csmc_run(hp.net, q, seed, first_run, n_runs, hp.d_flags, hp.d_values, steps ? hp.d_steps : nullptr, out,
                  hp.stream);
    if (rc || !n_runs) return rc;
    if (flags) {
        rc = copy_back(hp, hp.d_flags, 1, n_runs, flags, [](const void *, uint64_t, uint64_t) {});
        if (rc) return rc;
    }
    if (steps) {
        rc = copy_back(hp, hp.d_steps, sizeof(uint32_t), n_runs, steps, [](const void *, uint64_t, uint64_t) {});
        if (rc) return rc;
    }
    // values: always read back (the run-order sums need them); kept when the
    // caller passed a buffer
    double s = 0.0, s2 = 0.0;
    rc = copy_back(hp, hp.d_values, sizeof(double), n_runs, values, [&](const void *chunk, uint64_t cnt, uint64_t) {
        const double *v = static_cast<const double *>(chunk);
        for (uint64_t i = 0; i < cnt; ++i) {
            s += v[i];
            s2 += v[i] * v[i];
        }
    });
    if (rc) return rc;
    out->sum = s;
    out->sum_sq = s2;
    if (q->kind == CSMC_QUERY_VARIABLE && q->is_estimate) out->estimate = s / static_cast<double>(n_runs);
    return CSMC_OK;
}

}  // namespace

extern "C" {

int csmc_run_host(const void *blob, size_t bytes, const csmc_query *q, uint64_t seed, uint64_t first_run,
                  uint64_t n_runs, uint8_t *flags, double *values, uint32_t *steps, csmc_result *out) {
    try {
        return run_host(blob, bytes, q, seed, first_run, n_runs, flags, values, steps, out);
    } catch (const std::exception &e) {
        return fail(CSMC_ERR_ARG, e.what());
    }
}

void csmc_run_host_release(void) {
    std::lock_guard<std::mutex> lock(g_paths_mu);
    int cur = -1;
    cudaGetDevice(&cur);
    for (int d = 0; d < kMaxDevices; ++d) {
        if (!g_paths[d]) continue;
        std::lock_guard<std::mutex> l2(g_paths[d]->mu);
        if (cudaSetDevice(d) == cudaSuccess) g_paths[d]->release();
    }
    if (cur >= 0) cudaSetDevice(cur);
    cudaGetLastError();
}

}  // extern "C"
