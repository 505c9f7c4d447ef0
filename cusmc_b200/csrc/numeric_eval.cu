// csmc_numeric_eval: the numeric primitives whose exact bits define a run —
// Philox4x32-10, the exponential delay and its float log2, the double
// log2/exp2/pow of the expression language, and the proposal network's
// exp2 and GELU — evaluated by the device code the kernels inline, over
// device arrays.  A host compares these bits with its own evaluation of the
// same definitions (the CPU oracle compiles the same headers) and with
// independent references (published Philox known-answer vectors, libm).
#include "../../include/csmc.h"
#include "include/csmc_mlp.h"
#include "include/csmc_numeric.h"

#include <cuda_runtime.h>

#include <string>

namespace csmc {
void set_last_error(const std::string &m);  // capi.cu
}

namespace {

__global__ void numeric_eval_kernel(int32_t fn, const void *a, const void *b, uint64_t n, void *out) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        switch (fn) {
        case CSMC_NUM_PHILOX: {
            const uint32_t *c = static_cast<const uint32_t *>(a) + 4 * i;
            const uint32_t *k = static_cast<const uint32_t *>(b) + 2 * i;
            const csmc::u32x4 r = csmc::philox4x32_10(csmc::u32x4{c[0], c[1], c[2], c[3]}, k[0], k[1]);
            uint32_t *o = static_cast<uint32_t *>(out) + 4 * i;
            o[0] = r.x;
            o[1] = r.y;
            o[2] = r.z;
            o[3] = r.w;
            break;
        }
        case CSMC_NUM_PHILOX_STEP: {
            const uint32_t *c = static_cast<const uint32_t *>(a) + 4 * i;
            const uint32_t *k = static_cast<const uint32_t *>(b) + 2 * i;
            const csmc::PhiloxKeys K = csmc::philox_keys(static_cast<uint64_t>(k[0]) | (static_cast<uint64_t>(k[1]) << 32));
            const csmc::PhiloxStep S = csmc::philox_step(K, c[0], static_cast<uint64_t>(c[2]) | (static_cast<uint64_t>(c[3]) << 32));
            const csmc::u32x4 r = csmc::philox_block(K, S, c[1]);
            uint32_t *o = static_cast<uint32_t *>(out) + 4 * i;
            o[0] = r.x;
            o[1] = r.y;
            o[2] = r.z;
            o[3] = r.w;
            break;
        }
        case CSMC_NUM_EXP_DELAY:
            static_cast<float *>(out)[i] =
                csmc::exp_delay(static_cast<const uint32_t *>(a)[i], static_cast<const float *>(b)[i]);
            break;
        case CSMC_NUM_LOG2_F32:
            static_cast<float *>(out)[i] = csmc::log2_pos(static_cast<const float *>(a)[i]);
            break;
        case CSMC_NUM_LOG2_F64:
            static_cast<double *>(out)[i] = csmc::log2_d(static_cast<const double *>(a)[i]);
            break;
        case CSMC_NUM_EXP2_F64:
            static_cast<double *>(out)[i] = csmc::exp2_d(static_cast<const double *>(a)[i]);
            break;
        case CSMC_NUM_POW_F64:
            static_cast<double *>(out)[i] =
                csmc::pow_model(static_cast<const double *>(a)[i], static_cast<const double *>(b)[i]);
            break;
        case CSMC_NUM_EXP2_F32:
            static_cast<float *>(out)[i] = csmc::exp2_f(static_cast<const float *>(a)[i]);
            break;
        case CSMC_NUM_GELU_F32:
            static_cast<float *>(out)[i] = csmc::gelu_f(static_cast<const float *>(a)[i]);
            break;
        case CSMC_NUM_GELU_GRAD_F32:
            static_cast<float *>(out)[i] = csmc::gelu_grad_f(static_cast<const float *>(a)[i]);
            break;
        default:
            break;
        }
    }
}

}  // namespace

extern "C" int csmc_numeric_eval(int32_t fn, const void *a, const void *b, uint64_t n, void *out, void *stream) {
    if (fn < CSMC_NUM_PHILOX || fn > CSMC_NUM_PHILOX_STEP) {
        csmc::set_last_error("unknown numeric function " + std::to_string(fn));
        return CSMC_ERR_ARG;
    }
    const bool two = fn == CSMC_NUM_PHILOX || fn == CSMC_NUM_PHILOX_STEP || fn == CSMC_NUM_EXP_DELAY || fn == CSMC_NUM_POW_F64;
    if (n && (!a || !out || (two && !b))) {
        csmc::set_last_error("null argument");
        return CSMC_ERR_ARG;
    }
    if (!n) return CSMC_OK;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) {
        const uint64_t want = (n + 255) / 256, cap = static_cast<uint64_t>(sms) * 8;
        const int grid = static_cast<int>(want < cap ? want : cap);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        numeric_eval_kernel<<<grid, 256, 0, st>>>(fn, a, b, n, out);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        csmc::set_last_error(std::string("csmc_numeric_eval: ") + cudaGetErrorString(e));
        return CSMC_ERR_CUDA;
    }
    return CSMC_OK;
}
