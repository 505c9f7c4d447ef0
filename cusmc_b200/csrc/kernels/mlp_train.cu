// Tensor-core (tcgen05) kernels of the proposal network: the forward pass
// over a row set, and the gradient of the CE objective
//     J = sum over rows of (b * theta - a * e^theta)
// with respect to every parameter, both with BF16 operands and FP32
// accumulation in tensor memory.
//
// One CTA of 512 threads (four warpgroups) walks row tiles of 128 rows.
// Thread (g, r), g = warpgroup, r = thread index within it, owns row r of
// the tile (TMEM lane r; warp w reads TMEM lanes 32 (w mod 4) ..) and columns
// 16 g .. 16 g + 15 of each 64-wide layer, so the CUDA-core epilogues (GELU,
// GELU', the BF16 repacking) are spread over 16 warps.  Per tile:
//   D1 = X  . W1^T          (M=128, N=64,  K=16)   first layer
//   D2 = H1 . W2^T          (M=128, N=64,  K=64)   second layer
//   D1 = dZ2 . W2           (M=128, N=64,  K=64)   back-propagation into layer 1
//   D4 += [dZ2 | dZ1]^T . [H1 | X | 1]   (M=128, N=96, K=128 rows)
// so D4 accumulates dW2^T, dW1^T and the bias gradients over every tile the
// CTA processes.  A row's theta is the sum of its four groups' partial dot
// products (exchanged through shared memory, added in group order); the
// GELU derivatives stay in the registers of the thread that computed them,
// and the output layer's gradient is accumulated per thread in registers
// and reduced once at the end in a fixed order (the gradient is
// deterministic).  Operands live in shared memory in the no-swizzle K-major
// canonical layout (8-row x 16-byte core matrices; core matrix (row group g,
// K chunk c) at ((c * rows/8) + g) * 128 bytes), one thread issues the MMAs,
// completion is signalled through an mbarrier, and every wait is bounded: on
// a timeout the kernel records an error, waits (bounded) for its MMAs, frees
// its tensor memory and returns.
#include "../include/csmc_mlp.h"
#include "sim.cuh"

#include <cuda_runtime.h>

namespace csmc {
namespace {

constexpr int kRows = 128;                      // rows per tile
constexpr int kGroups = 4;                      // warpgroups per CTA
constexpr int kThreads = 128 * kGroups;
constexpr int kCols = CSMC_MLP_HID / kGroups;   // layer columns per thread (16)
constexpr uint32_t kTmemCols = 256;             // D1/D3 [0,64), D2 [64,128), D4 [128,224)
constexpr uint32_t kColD1 = 0, kColD2 = 64, kColD4 = 128;
constexpr int kN4 = 96;                         // [H1 (64) | X (16) | 1 | 0 x 15]

// shared-memory carve-up (bytes).  The dZ2 tile (A3) reuses the H1 tile's
// space (A2): the layer-2 MMA that reads A2 has completed before the
// epilogue writes A3, and the next tile writes A2 only after the MMA that
// reads A3 has completed.  The allocation extends far beyond the last
// operand tile (kSmemBytes), so operand accesses stay inside it even under a
// transposed reading of the descriptor strides.
constexpr uint32_t kA1 = 0;                     // X tile      128 x 16
constexpr uint32_t kB1 = kA1 + 128 * 16 * 2;    // W1          64 x 16
constexpr uint32_t kA2 = kB1 + 64 * 16 * 2;     // H1 tile     128 x 64; later dZ2 (A3)
constexpr uint32_t kA3 = kA2;
constexpr uint32_t kB2 = kA2 + 128 * 64 * 2;    // W2          64 x 64 (out x in)
constexpr uint32_t kB3 = kB2 + 64 * 64 * 2;     // W2^T        64 x 64 (in x out)
constexpr uint32_t kA4 = kB3 + 64 * 64 * 2;     // dZ^T        128 x 128 (neuron x row)
constexpr uint32_t kB4 = kA4 + 128 * 128 * 2;   // F^T         96 x 128 (feature x row)
constexpr uint32_t kTh = kB4 + kN4 * 128 * 2;   // theta partials [group][row] (floats)
constexpr uint32_t kMisc = kTh + kGroups * 128 * 4;  // mbarrier, tmem address, biases, reductions
constexpr uint32_t kMiscBytes = 4096;
constexpr uint32_t kRedStride = 17;             // per-warp output-layer sums: 16 columns, db3
constexpr uint32_t kSmemBytes = 160 * 1024;     // >= the operands' extent under either stride reading
static_assert(kMisc + kMiscBytes <= kSmemBytes, "shared-memory carve-up");
static_assert(1536 + 16 * kRedStride * 4 <= kMiscBytes, "reduction slots");

constexpr uint32_t kWaitLimit = 1u << 20;       // bounded mbarrier polls

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) in a K-major no-swizzle tile of R rows
__device__ __forceinline__ uint32_t kmaj(uint32_t r, uint32_t k, uint32_t R) {
    return (((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7u) << 4) + ((k & 7u) << 1);
}

// shared-memory matrix descriptor: start, leading (K) and stride (row
// group) byte offsets, version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((addr >> 4) & 0x3fffu) | (static_cast<uint64_t>((lbo >> 4) & 0x3fffu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M=128
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;  // no output lane disabled
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void st_bf16(uint8_t *base, uint32_t off, float v) {
    *reinterpret_cast<uint16_t *>(base + off) = f_to_bf16(v);
}

// Waits for the MMAs committed to mbar, block-uniformly: false when any
// thread's bounded wait gave up.
__device__ __forceinline__ bool wait_all(uint32_t mbar, uint32_t &phase) {
    const int mine = mbar_wait(mbar, phase) ? 1 : 0;
    phase ^= 1u;
    const bool all = __syncthreads_and(mine) != 0;
    tc_after_sync();
    return all;
}

// mode 0: forward only (clipped theta per row into theta_out); mode 1:
// gradient partials per CTA: D4 (128 x 96 floats: row m = output neuron of
// [layer 2 | layer 1], column n = input [h1 | x | 1 | 0]), dw3 (64), db3, 0.
template <int MODE>
__global__ void __launch_bounds__(kThreads, 1)
    mlp_tc_kernel(const MlpRow *rows, uint64_t n_rows, const MlpParams *P, float *theta_out, float *partials,
                  double *objective, int *error) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t grp = tid >> 7, r = tid & 127u;  // warpgroup, row within the tile
    const uint32_t c0 = grp * kCols;                // this thread's first layer column
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + kMisc);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(sm + kMisc + 8);
    float *b1s = reinterpret_cast<float *>(sm + kMisc + 512);
    float *b2s = reinterpret_cast<float *>(sm + kMisc + 768);
    float *w3s = reinterpret_cast<float *>(sm + kMisc + 1024);
    float *red = reinterpret_cast<float *>(sm + kMisc + 1536);  // [warp][kRedStride]
    float *thp = reinterpret_cast<float *>(sm + kTh);           // [group][row]
    const uint32_t mbar_a = smem_u32(mbar);

    // ---- constant operands: W1 (B1), W2 (B2), W2^T (B3), the ones column of B4
    for (uint32_t i = tid; i < 64 * 16; i += blockDim.x) {
        const uint32_t o = i / 16, in = i % 16;
        *reinterpret_cast<uint16_t *>(sm + kB1 + kmaj(o, in, 64)) = P->w1[o][in];
    }
    for (uint32_t i = tid; i < 64 * 64; i += blockDim.x) {
        const uint32_t o = i / 64, in = i % 64;
        *reinterpret_cast<uint16_t *>(sm + kB2 + kmaj(o, in, 64)) = P->w2[o][in];
        *reinterpret_cast<uint16_t *>(sm + kB3 + kmaj(in, o, 64)) = P->w2[o][in];
    }
    for (uint32_t nn = 80 + grp * 4; nn < 84 + grp * 4; ++nn) st_bf16(sm + kB4, kmaj(nn, r, kN4), nn == 80 ? 1.0f : 0.0f);
    if (tid < 64) {
        b1s[tid] = P->b1[tid];
        b2s[tid] = P->b2[tid];
        w3s[tid] = P->w3[tid];
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tmem_holder;
    const uint32_t lane_base = ((warp & 3u) * 32u) << 16;  // this warp's TMEM lanes (rows)
    const float b3 = P->b3;
    double J = 0.0;
    float dw3[kCols];  // this thread's rows' g * h2 for its columns, over all tiles
#pragma unroll
    for (int i = 0; i < kCols; ++i) dw3[i] = 0.0f;
    float db3 = 0.0f;
    uint32_t phase = 0;
    bool ok = true, first = true;

    const uint64_t tiles = (n_rows + kRows - 1) / kRows;
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint64_t row_i = tile * kRows + r;
        const bool valid = row_i < n_rows;
        MlpRow row;
        if (valid) {
            row = rows[row_i];
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) row.x[i] = 0;
            row.a = row.b = 0.0f;
        }
        // each group stores four of the row's sixteen features
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t f = grp * 4u + i;
            *reinterpret_cast<uint16_t *>(sm + kA1 + kmaj(r, f, kRows)) = row.x[f];
            if (MODE == 1) *reinterpret_cast<uint16_t *>(sm + kB4 + kmaj(64 + f, r, kN4)) = row.x[f];
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        // ---- layer 1
        if (tid == 0) {
            tc_after_sync();
            mma_bf16(tmem + kColD1, sdesc(smem_u32(sm + kA1), 2048, 128), sdesc(smem_u32(sm + kB1), 1024, 128),
                     idesc_bf16(64), 0);
            mma_commit(mbar_a);
        }
        if (!(ok = wait_all(mbar_a, phase))) break;
        float dg1[kCols];  // GELU'(z1) of this thread's columns
        {
            float z[16];
            tmem_ld16(tmem + lane_base + kColD1 + c0, z);
#pragma unroll
            for (int i = 0; i < kCols; ++i) {
                const uint32_t j = c0 + i;
                float gv;
                gelu_both(f_add(z[i], b1s[j]), gv, dg1[i]);
                const float h = bf16_round(gv);
                st_bf16(sm + kA2, kmaj(r, j, kRows), h);
                if (MODE == 1) st_bf16(sm + kB4, kmaj(j, r, kN4), h);
            }
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        // ---- layer 2
        if (tid == 0) {
            tc_after_sync();
#pragma unroll
            for (uint32_t kk = 0; kk < 4; ++kk)
                mma_bf16(tmem + kColD2, sdesc(smem_u32(sm + kA2 + kk * 4096), 2048, 128),
                         sdesc(smem_u32(sm + kB2 + kk * 2048), 1024, 128), idesc_bf16(64), kk > 0);
            mma_commit(mbar_a);
        }
        if (!(ok = wait_all(mbar_a, phase))) break;
        float h2[kCols], dg2[kCols];
        {
            float z2[16];
            tmem_ld16(tmem + lane_base + kColD2 + c0, z2);
            float part = 0.0f;
#pragma unroll
            for (int i = 0; i < kCols; ++i) {
                gelu_both(f_add(z2[i], b2s[c0 + i]), h2[i], dg2[i]);
                part = f_fma(h2[i], w3s[c0 + i], part);
            }
            thp[grp * 128 + r] = part;
        }
        __syncthreads();
        const float th = f_add(f_add(f_add(f_add(b3, thp[r]), thp[128 + r]), thp[256 + r]), thp[384 + r]);
        const bool inside = th >= -CSMC_MLP_THETA_MAX && th <= CSMC_MLP_THETA_MAX;
        const float thc = inside ? th : (th < 0.0f ? -CSMC_MLP_THETA_MAX : CSMC_MLP_THETA_MAX);
        if (MODE == 0) {
            if (valid && grp == 0) theta_out[row_i] = thc;
            tc_before_sync();
            __syncthreads();
            continue;
        }
        const float e = exp2_f(f_mul(thc, 1.44269502f));
        if (valid && grp == 0) J += static_cast<double>(row.b) * thc - static_cast<double>(row.a) * e;
        const float g = (valid && inside) ? f_add(row.b, -f_mul(row.a, e)) : 0.0f;
        if (grp == 0) db3 = f_add(db3, g);
#pragma unroll
        for (int i = 0; i < kCols; ++i) {
            const uint32_t k = c0 + i;
            dw3[i] = f_fma(g, h2[i], dw3[i]);
            const float dz = f_mul(f_mul(g, w3s[k]), dg2[i]);
            st_bf16(sm + kA3, kmaj(r, k, kRows), dz);
            st_bf16(sm + kA4, kmaj(k, r, kRows), dz);
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        // ---- back-propagation into the first layer: dH1 = dZ2 . W2
        if (tid == 0) {
            tc_after_sync();
#pragma unroll
            for (uint32_t kk = 0; kk < 4; ++kk)
                mma_bf16(tmem + kColD1, sdesc(smem_u32(sm + kA3 + kk * 4096), 2048, 128),
                         sdesc(smem_u32(sm + kB3 + kk * 2048), 1024, 128), idesc_bf16(64), kk > 0);
            mma_commit(mbar_a);
        }
        if (!(ok = wait_all(mbar_a, phase))) break;
        {
            float dh[16];
            tmem_ld16(tmem + lane_base + kColD1 + c0, dh);
#pragma unroll
            for (int i = 0; i < kCols; ++i) st_bf16(sm + kA4, kmaj(64 + c0 + i, r, kRows), f_mul(dh[i], dg1[i]));
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        // ---- weight gradients: D4 += dZ^T . F
        if (tid == 0) {
            tc_after_sync();
#pragma unroll
            for (uint32_t kk = 0; kk < 8; ++kk)
                mma_bf16(tmem + kColD4, sdesc(smem_u32(sm + kA4 + kk * 4096), 2048, 128),
                         sdesc(smem_u32(sm + kB4 + kk * 3072), 1536, 128), idesc_bf16(kN4), (!first || kk > 0));
            mma_commit(mbar_a);
        }
        first = false;
        if (!(ok = wait_all(mbar_a, phase))) break;
    }
    if (!ok) {
        if (error) atomicExch(error, 1);
        // one more bounded wait for the MMAs still in flight before freeing
        (void)mbar_wait(mbar_a, phase ^ 1u);
    }

    if (MODE == 1) {
        float *out = partials + static_cast<size_t>(blockIdx.x) * (128 * kN4 + 66);
        if (grp < 3) {  // groups 0..2 read 32 of D4's 96 columns each
            if (ok && !first) {  // block-uniform
                float v[16];
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const uint32_t col = grp * 32u + 16u * c;
                    tmem_ld16(tmem + lane_base + kColD4 + col, v);
#pragma unroll
                    for (int i = 0; i < 16; ++i) out[r * kN4 + col + i] = v[i];
                }
            } else {
                for (int i = 0; i < 32; ++i) out[r * kN4 + grp * 32 + i] = 0.0f;
            }
        }
        // output layer: per warp, the sum over its 32 rows (butterfly), then
        // the four warps of a group in warp order
#pragma unroll
        for (int i = 0; i < kCols; ++i) {
            float v = dw3[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp * kRedStride + i] = v;
        }
        float vb = db3;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vb += __shfl_xor_sync(0xffffffffu, vb, o);
        if (lane == 0) red[warp * kRedStride + kCols] = vb;
        __syncthreads();
        if (tid < 64) {  // dw3[k]: group k / 16, its warps 4g .. 4g + 3
            const uint32_t gk = tid / kCols, i = tid % kCols;
            const float *rw = red + (4 * gk) * kRedStride + i;
            out[128 * kN4 + tid] =
                f_add(f_add(f_add(rw[0], rw[kRedStride]), rw[2 * kRedStride]), rw[3 * kRedStride]);
        }
        if (tid == 64)
            out[128 * kN4 + 64] = f_add(f_add(f_add(red[kCols], red[kRedStride + kCols]), red[2 * kRedStride + kCols]),
                                        red[3 * kRedStride + kCols]);
        if (tid == 65) out[128 * kN4 + 65] = 0.0f;
        __shared__ double jred[128];
        if (grp == 0) jred[r] = J;
        __syncthreads();
        if (tid == 0) {
            double sum = 0.0;
            for (int i = 0; i < 128; ++i) sum += jred[i];
            objective[blockIdx.x] = sum;
        }
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

size_t mlp_tc_smem_bytes() { return kSmemBytes; }
int mlp_tc_partial_floats() { return 128 * kN4 + 66; }

int mlp_tc_launch(int mode, const MlpRow *rows, uint64_t n_rows, const MlpParams *P, float *theta_out,
                  float *partials, double *objective, int *error, int grid, void *stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (mode == 0) {
        auto fn = mlp_tc_kernel<0>;
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        if (e != cudaSuccess) return static_cast<int>(e);
        fn<<<grid, kThreads, kSmemBytes, st>>>(rows, n_rows, P, theta_out, partials, objective, error);
    } else {
        auto fn = mlp_tc_kernel<1>;
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        if (e != cudaSuccess) return static_cast<int>(e);
        fn<<<grid, kThreads, kSmemBytes, st>>>(rows, n_rows, P, theta_out, partials, objective, error);
    }
    return static_cast<int>(cudaGetLastError());
}

}  // namespace csmc
