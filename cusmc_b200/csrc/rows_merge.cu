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

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kChainsPerBlock = 4;  // one warp per chain, 128 threads per CTA

// Walks chain c (run i = c / 4, class l = c % 4: rows off[i] + l, + 4, ...,
// below the next run's first row) with one warp, 32 consecutive steps per
// batch, lane j holding step s0 + j.  A step starts a group when it is the
// chain's first or its features differ from the previous step's (which,
// within a group, equal the group's first row's).  Each group's a and b are
// summed in FP64 in step order from 0.0 by the lane of its first step in
// the batch, which for a group begun in an earlier batch is lane 0
// continuing the carried sums (a group beginning on lane 0 instead closes
// the carried one): the same additions in the same order as one thread
// walking the chain.  emit(j, first row, a, b) runs, on one lane, for
// each group whose sums are not both zero, j counting those groups in step
// order; returns their number (on every lane).  sh: this warp's 64 floats of
// shared memory.
template <class Emit>
__device__ __forceinline__ uint32_t walk_chain(const uint32_t *rows, const uint64_t *off, uint64_t n_list,
                                               uint64_t n_rows, uint64_t c, float *sh, Emit emit) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t i = c >> 2;
    const uint64_t first = off[i] + (c & 3u);
    uint64_t end = i + 1 < n_list ? off[i + 1] : n_rows;
    if (end > n_rows) end = n_rows;
    const uint64_t len = end > first ? (end - first + 3) / 4 : 0;
    uint32_t prev[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // the previous batch's last row's features
    double ca = 0.0, cb = 0.0;                       // sums of the group open at the batch boundary
    uint64_t chead = 0;                              // its first row
    uint32_t groups = 0;
    for (uint64_t s0 = 0; s0 < len; s0 += 32) {
        const uint64_t s = s0 + lane;
        const bool valid = s < len;
        const uint32_t nvalid = len - s0 < 32 ? static_cast<uint32_t>(len - s0) : 32u;
        const uint64_t r = first + 4 * s;
        uint32_t w[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) w[k] = valid ? rows[r * kRowWords + k] : 0u;
        bool same = true;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            uint32_t pk = __shfl_up_sync(kFull, w[k], 1);
            if (lane == 0) pk = prev[k];
            same = same && w[k] == pk;
        }
        const bool head = valid && (s == 0 || !same);
        // a group beginning on lane 0 closes the group carried over
        if (s0 > 0 && (__ballot_sync(kFull, head) & 1u) && (ca != 0.0 || cb != 0.0)) {
            if (lane == 0) emit(groups, chead, ca, cb);
            ++groups;
        }
        sh[lane] = __uint_as_float(w[8]);
        sh[32 + lane] = __uint_as_float(w[9]);
        __syncwarp();
        const bool start = valid && (head || lane == 0);
        const uint32_t S = __ballot_sync(kFull, start);
        const uint32_t later = lane < 31 ? S & ~((2u << lane) - 1u) : 0u;
        const uint32_t seg_end = later ? static_cast<uint32_t>(__ffs(later) - 1) : nvalid;
        double sa = 0.0, sb = 0.0;
        uint64_t hr = r;
        if (start && !head) {  // lane 0 continuing the carried group
            sa = ca;
            sb = cb;
            hr = chead;
        }
        if (start)
            for (uint32_t t = lane; t < seg_end; ++t) {
                sa = csmc::d_add(sa, static_cast<double>(sh[t]));
                sb = csmc::d_add(sb, static_cast<double>(sh[32 + t]));
            }
        // the batch's last group stays open unless the chain ends here
        const bool complete = start && (seg_end < nvalid || s0 + 32 >= len);
        const bool emits = complete && (sa != 0.0 || sb != 0.0);
        const uint32_t E = __ballot_sync(kFull, emits);
        if (emits) emit(groups + __popc(E & ((1u << lane) - 1u)), hr, sa, sb);
        groups += __popc(E);
        const int src = 31 - __clz(S);  // lane 0 always starts a segment
        ca = __shfl_sync(kFull, sa, src);
        cb = __shfl_sync(kFull, sb, src);
        chead = __shfl_sync(kFull, hr, src);
#pragma unroll
        for (int k = 0; k < 8; ++k) prev[k] = __shfl_sync(kFull, w[k], static_cast<int>(nvalid) - 1);
        __syncwarp();  // sh is rewritten by the next batch
    }
    return groups;
}

__global__ void merge_count(const uint32_t *rows, const uint64_t *off, uint64_t n_list, uint64_t n_rows,
                            uint32_t *counts) {
    __shared__ float sh[kChainsPerBlock][64];
    const uint32_t wi = threadIdx.x >> 5;
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * kChainsPerBlock + wi;
    if (c >= 4 * n_list) return;  // whole warps
    const uint32_t g =
        walk_chain(rows, off, n_list, n_rows, c, sh[wi], [](uint32_t, uint64_t, double, double) {});
    if ((threadIdx.x & 31u) == 0) counts[c] = g;
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
    __shared__ float sh[kChainsPerBlock][64];
    const uint32_t wi = threadIdx.x >> 5;
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * kChainsPerBlock + wi;
    if (c >= 4 * n_list) return;  // whole warps
    const uint64_t b = base[c];
    walk_chain(rows, off, n_list, n_rows, c, sh[wi], [&](uint32_t j, uint64_t head, double sa, double sb) {
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
    const unsigned blocks = static_cast<unsigned>((chains + kChainsPerBlock - 1) / kChainsPerBlock);
    merge_count<<<blocks, 32 * kChainsPerBlock, 0, st>>>(r, row_offset, n_list, n_rows, m.counts);
    CK(cudaGetLastError(), "row-merge count launch");
    merge_scan<<<1, 1024, 0, st>>>(m.counts, chains, m.base);
    CK(cudaGetLastError(), "row-merge scan launch");
    merge_write<<<blocks, 32 * kChainsPerBlock, 0, st>>>(r, row_offset, n_list, n_rows, m.base,
                                                         static_cast<uint32_t *>(out));
    CK(cudaGetLastError(), "row-merge write launch");
    uint64_t total = 0;
    CK(cudaMemcpyAsync(&total, m.base + chains, sizeof total, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    CK(cudaStreamSynchronize(st), "row merge");
    *n_out = total;
    return CSMC_OK;
}

}  // extern "C"
