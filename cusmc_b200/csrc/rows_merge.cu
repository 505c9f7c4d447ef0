// Merging of CE training rows (csmc_mlp_rows_merge).
//
// A replayed run writes four rows per step, one per location class.  The
// CE objective J = sum over rows of (b theta(x) - a e^theta(x)) is linear in
// (a, b) for a fixed feature row x, so consecutive steps of one run whose
// rows of a class carry the same features (steps in which no variable
// changed and time stayed within one step of the time feature, the majority
// of an epidemic run's steps) can be summed into one row without changing J
// or its gradient in exact arithmetic.  Within a run and a class, rows are
// grouped by equal features in step order; a group's a and b are summed in
// FP64 in step order and rounded to FP32; groups whose a and b are both
// zero (nothing of the class was tilted, or nothing fired) carry no term
// and are dropped.  Output order: run, class, first step of the group.
#include "../../include/csmc.h"
#include "capi_internal.h"
#include "include/csmc_mlp.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

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

constexpr uint32_t kRowWords = sizeof(csmc::MlpRow) / 4;  // 8 words of features, then a and b
static_assert(sizeof(csmc::MlpRow) == 40, "row layout: 16 BF16 features, two floats");

// Walks the chain of rows of run i, class l (rows off[i] + l, + 4, ...,
// below the next run's first row) and hands each nonzero group to emit(j,
// first row, a, b), j counting the chain's groups.
template <class Emit>
__device__ __forceinline__ uint32_t walk_chain(const uint32_t *rows, const uint64_t *off, uint64_t n_list,
                                               uint64_t n_rows, uint64_t c, Emit emit) {
    const uint64_t i = c >> 2;
    const uint64_t end = i + 1 < n_list ? off[i + 1] : n_rows;
    uint32_t key[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t head = 0;
    bool open = false;
    double sa = 0.0, sb = 0.0;
    uint32_t groups = 0;
    for (uint64_t r = off[i] + (c & 3u); r < end; r += 4) {
        const uint32_t *w = rows + r * kRowWords;
        bool same = open;
#pragma unroll
        for (int j = 0; j < 8; ++j) same = same && w[j] == key[j];
        if (!same) {
            if (open && (sa != 0.0 || sb != 0.0)) emit(groups++, head, sa, sb);
#pragma unroll
            for (int j = 0; j < 8; ++j) key[j] = w[j];
            head = r;
            sa = sb = 0.0;
            open = true;
        }
        sa = csmc::d_add(sa, static_cast<double>(__uint_as_float(w[8])));
        sb = csmc::d_add(sb, static_cast<double>(__uint_as_float(w[9])));
    }
    if (open && (sa != 0.0 || sb != 0.0)) emit(groups++, head, sa, sb);
    return groups;
}

__global__ void merge_count(const uint32_t *rows, const uint64_t *off, uint64_t n_list, uint64_t n_rows,
                            uint32_t *counts) {
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= 4 * n_list) return;
    counts[c] = walk_chain(rows, off, n_list, n_rows, c, [](uint32_t, uint64_t, double, double) {});
}

// Exclusive prefix sums of m counts in one CTA of 1024 threads (each thread
// a contiguous segment); base[m] = the total.
__global__ void merge_scan(const uint32_t *counts, uint64_t m, uint64_t *base) {
    __shared__ uint64_t part[1024];
    const uint64_t seg = (m + blockDim.x - 1) / blockDim.x;
    const uint64_t b = threadIdx.x * seg, e = b + seg < m ? b + seg : m;
    uint64_t s = 0;
    for (uint64_t k = b; k < e; ++k) s += counts[k];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t run = 0;
        for (uint32_t t = 0; t < blockDim.x; ++t) {
            const uint64_t v = part[t];
            part[t] = run;
            run += v;
        }
        base[m] = run;
    }
    __syncthreads();
    uint64_t run = part[threadIdx.x];
    for (uint64_t k = b; k < e; ++k) {
        base[k] = run;
        run += counts[k];
    }
}

__global__ void merge_write(const uint32_t *rows, const uint64_t *off, uint64_t n_list, uint64_t n_rows,
                            const uint64_t *base, uint32_t *out) {
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= 4 * n_list) return;
    const uint64_t b = base[c];
    walk_chain(rows, off, n_list, n_rows, c, [&](uint32_t j, uint64_t head, double sa, double sb) {
        uint32_t *o = out + (b + j) * kRowWords;
        const uint32_t *w = rows + head * kRowWords;
#pragma unroll
        for (int k = 0; k < 8; ++k) o[k] = w[k];
        o[8] = __float_as_uint(static_cast<float>(sa));
        o[9] = __float_as_uint(static_cast<float>(sb));
    });
}

// Per-device scratch (counts and their prefix sums), kept for the life of
// the process.
struct MergeScratch {
    std::mutex mu;
    uint32_t *counts = nullptr;
    uint64_t *base = nullptr;
    uint64_t cap = 0;
};

MergeScratch &merge_scratch(int dev) {
    static MergeScratch sets[64];
    return sets[dev & 63];
}

}  // namespace

extern "C" {

int csmc_mlp_rows_merge(const void *rows, const uint64_t *row_offset, uint64_t n_list, uint64_t n_rows, void *out,
                        uint64_t *n_out, void *stream) {
    if (!n_out || (n_rows && (!rows || !row_offset || !out))) return fail(CSMC_ERR_ARG, "null argument");
    *n_out = 0;
    if (n_list == 0 || n_rows == 0) return CSMC_OK;
    int dev = 0;
    CK(cudaGetDevice(&dev), "cudaGetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MergeScratch &m = merge_scratch(dev);
    std::lock_guard<std::mutex> lock(m.mu);
    const uint64_t chains = 4 * n_list;
    if (chains > m.cap) {
        cudaFree(m.counts);
        cudaFree(m.base);
        m.counts = nullptr;
        m.base = nullptr;
        m.cap = 0;
        CK(cudaMalloc(&m.counts, chains * sizeof(uint32_t)), "cudaMalloc(row-merge counts)");
        CK(cudaMalloc(&m.base, (chains + 1) * sizeof(uint64_t)), "cudaMalloc(row-merge offsets)");
        m.cap = chains;
    }
    const uint32_t *r = static_cast<const uint32_t *>(rows);
    const unsigned blocks = static_cast<unsigned>((chains + 127) / 128);
    merge_count<<<blocks, 128, 0, st>>>(r, row_offset, n_list, n_rows, m.counts);
    CK(cudaGetLastError(), "row-merge count launch");
    merge_scan<<<1, 1024, 0, st>>>(m.counts, chains, m.base);
    CK(cudaGetLastError(), "row-merge scan launch");
    merge_write<<<blocks, 128, 0, st>>>(r, row_offset, n_list, n_rows, m.base, static_cast<uint32_t *>(out));
    CK(cudaGetLastError(), "row-merge write launch");
    uint64_t total = 0;
    CK(cudaMemcpyAsync(&total, m.base + chains, sizeof total, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CK(cudaStreamSynchronize(st), "row merge");
    *n_out = total;
    return CSMC_OK;
}

}  // extern "C"
