// csmc_measure_smem_bandwidth: the shared-memory bandwidth of the current
// device, measured.  The thread-per-run simulation kernel is bound by
// shared-memory and issue throughput rather than HBM, so its roofline needs
// a shared-memory peak; this kernel gives a measured one instead of the
// data-sheet figure (128 B per clock per SM).
//
// Every CTA streams 16-byte loads from a 16 KB shared buffer, a warp reading
// 512 consecutive bytes per load (four 128-byte wavefronts, no bank
// conflicts), eight independent loads in flight per thread.  Each CTA also
// records clock64() and %globaltimer around its loop, which gives the SM
// clock during the measurement.
#include "../../include/csmc.h"

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace csmc {
void set_last_error(const std::string &m);  // capi.cu
}

namespace {

constexpr int kProbeBlock = 256;
constexpr int kProbeWords = 1024;  // uint4 words: 16 KB per CTA
constexpr int kProbeUnroll = 8;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void __launch_bounds__(kProbeBlock) smem_stream_kernel(uint32_t iters, uint32_t *sink,
                                                                  unsigned long long *clk) {
    __shared__ __align__(16) uint4 buf[kProbeWords];
    for (int i = threadIdx.x; i < kProbeWords; i += blockDim.x)
        buf[i] = make_uint4(i, i * 3u + 1u, i * 5u + 2u, i * 7u + 3u);
    __syncthreads();
    const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(buf));
    uint32_t acc[kProbeUnroll];
#pragma unroll
    for (int u = 0; u < kProbeUnroll; ++u) acc[u] = 0;
    const unsigned long long c0 = clock64(), t0 = global_ns();
    for (uint32_t it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < kProbeUnroll; ++u) {
            // word index: this warp's 32 consecutive words, rotated per load
            const uint32_t w = (threadIdx.x + (it * kProbeUnroll + u) * 32u) & (kProbeWords - 1);
            uint32_t a, b, c, d;
            asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                         : "=r"(a), "=r"(b), "=r"(c), "=r"(d)
                         : "r"(base + 16u * w));
            acc[u] ^= a ^ b ^ c ^ d;
        }
    }
    const unsigned long long c1 = clock64(), t1 = global_ns();
    uint32_t x = 0;
#pragma unroll
    for (int u = 0; u < kProbeUnroll; ++u) x ^= acc[u];
    if (x == 0x9e3779b9u) sink[0] = x;  // keeps the loads alive
    if (threadIdx.x == 0) {
        clk[2 * blockIdx.x] = c1 - c0;
        clk[2 * blockIdx.x + 1] = t1 - t0;
    }
}

int fail(int code, const std::string &m) {
    csmc::set_last_error(m);
    return code;
}

}  // namespace

extern "C" int csmc_measure_smem_bandwidth(double *gbs, double *sm_mhz) {
    if (!gbs) return fail(CSMC_ERR_ARG, "null argument");
    int dev = 0, sms = 0, count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(CSMC_ERR_NODEVICE, "no CUDA device is available");
    }
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(CSMC_ERR_CUDA, std::string("device attributes: ") + cudaGetErrorString(e));
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, smem_stream_kernel, kProbeBlock, 0);
    if (e != cudaSuccess || per_sm < 1) return fail(CSMC_ERR_CUDA, "occupancy query of the shared-memory probe");
    const int grid = sms * per_sm;
    const uint32_t iters = 128;  // 16 KB per thread: ~5 GB of shared-memory reads per launch at 8 CTAs/SM
    uint32_t *d_sink = nullptr;
    unsigned long long *d_clk = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    auto cleanup = [&] {
        cudaFree(d_sink);
        cudaFree(d_clk);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    };
    e = cudaMalloc(&d_sink, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&d_clk, 2 * sizeof(unsigned long long) * grid);
    if (e == cudaSuccess) e = cudaEventCreate(&ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ev1);
    float best_ms = 0.0f;
    for (int rep = 0; e == cudaSuccess && rep < 4; ++rep) {  // the first launch warms up
        e = cudaEventRecord(ev0, nullptr);
        smem_stream_kernel<<<grid, kProbeBlock>>>(iters, d_sink, d_clk);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(ev1, nullptr);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev1);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev0, ev1);
        if (e == cudaSuccess && rep > 0 && (best_ms == 0.0f || ms < best_ms)) best_ms = ms;
    }
    std::vector<unsigned long long> clk(2 * static_cast<size_t>(grid));
    if (e == cudaSuccess)
        e = cudaMemcpy(clk.data(), d_clk, clk.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cleanup();
    if (e != cudaSuccess) return fail(CSMC_ERR_CUDA, std::string("shared-memory probe: ") + cudaGetErrorString(e));
    const double bytes = static_cast<double>(grid) * kProbeBlock * iters * kProbeUnroll * 16.0;
    *gbs = bytes / (best_ms / 1000.0) / 1e9;
    if (sm_mhz) {
        double cyc = 0.0, ns = 0.0;
        for (int b = 0; b < grid; ++b) {
            cyc += static_cast<double>(clk[2 * b]);
            ns += static_cast<double>(clk[2 * b + 1]);
        }
        *sm_mhz = ns > 0.0 ? 1000.0 * cyc / ns : 0.0;
    }
    return CSMC_OK;
}
