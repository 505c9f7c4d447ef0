// Deterministic sum and sum of squares of per-run values: fixed chunking
// into kReduceBlocks blocks of 256 threads, fixed per-thread order and a
// fixed shared-memory tree, so a job's sums do not depend on how or where
// its runs were simulated (the single-network and the batch paths give the
// same bits).
#pragma once
#include <cstdint>

#include "../include/csmc_numeric.h"

namespace csmc {

constexpr int kReduceBlocks = 256;

// Block `block` of the reduction of values[0..n) into out[0] (sum) and
// out[1] (sum of squares); 256 threads.
static __device__ __forceinline__ void reduce_block(const double *values, uint64_t n, uint32_t block, double *out) {
    __shared__ double s1[256], s2[256];
    const uint64_t chunk = (n + kReduceBlocks - 1) / kReduceBlocks;
    const uint64_t b0 = block * chunk, b1 = (b0 + chunk < n) ? b0 + chunk : n;
    double a = 0.0, q = 0.0;
    for (uint64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double v = values[i];
        a = d_add(a, v);
        q = d_add(q, d_mul(v, v));
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = q;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            s1[threadIdx.x] = d_add(s1[threadIdx.x], s1[threadIdx.x + s]);
            s2[threadIdx.x] = d_add(s2[threadIdx.x], s2[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s1[0];
        out[1] = s2[0];
    }
}

}  // namespace csmc
