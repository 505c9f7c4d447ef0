// Internal to libcsmc: the device network handle behind csmc_net (shared by
// capi.cu and capi_batch.cu).
#pragma once
#include "../../include/csmc.h"
#include "include/csmc_net.h"
#include "kernels/sim.cuh"

#include <cuda_runtime.h>

#include <string>

struct csmc_net {
    int device = 0;
    uint8_t *d_blob = nullptr;
    uint32_t bytes = 0;       // staged bytes (multiple of 16)
    csmc_net_header h{};
    unsigned long long *d_scratch = nullptr;
    // internal per-run buffers used when the caller passes none
    uint8_t *d_flags = nullptr;
    double *d_values = nullptr;
    uint64_t cap_runs = 0;
    double *d_partials = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // launch plan: family 0 = lane groups (lanes, comps_per_lane), 1 = one
    // thread per run, 2 = one thread per run with the network read from
    // global memory (the batch kernel with one job)
    int family = 1;
    int lanes = 0, comps_per_lane = 0, block = 256, grid = 0;
    size_t smem = 0;
    uint32_t state_stride = 0;
    bool slots = false;
    bool loc8 = false;     // every automaton has at most 256 locations
    bool classes = false;  // delay descriptors carry race classes
    bool all_classed = false;  // every location belongs to a race class
    uint32_t class_src[CSMC_RACE_CLASSES] = {};  // 1/rate source of each class (SimParams::class_src)
    bool state_in_global = false;
    uint8_t *d_state = nullptr;  // thread-per-run state slabs (global-state plans)
    size_t state_bytes = 0;
    csmc::BatchJob *d_job = nullptr;  // family 2: the one-job table
    // importance sampling
    csmc::MlpParams *d_mlp = nullptr;  // the proposal network
    double *d_wvals = nullptr;         // per run: flag * likelihood ratio
    uint8_t *d_is_flags = nullptr;
    uint64_t is_cap = 0;
    bool is_tc = false;  // importance sampling: theta by warp-level MMAs (false: the oracle-identical CUDA-core evaluation)
    bool is_feat_set = false;   // importance sampling: a feature source was chosen (else the default)
    csmc::MlpFeatures is_feat{};
    // importance sampling one thread per run (sim_is_coded.cuh): the tilt
    // groups of the network (is_groups < 0: the network does not qualify)
    int is_groups = -1;
    bool is_all_grouped = false;  // every location in a tilt group, components a multiple of 4
    uint64_t is_group_map = 0;
    uint32_t is_group_l = 0;
    uint32_t is_group_src[CSMC_IS_GROUPS] = {};
    int is_kernel = 0;  // 0: thread per run where the network qualifies, 3: always one warp per run
    uint32_t *d_theta_cache = nullptr;  // thread-per-run kernel: the device-wide theta cache
    uint32_t theta_gen = 0;             // generation of the cached parameter block (0: none yet)
    unsigned char theta_params[CSMC_MLP_PARAM_BYTES] = {};  // the parameter block of that generation
};

namespace csmc {
void set_last_error(const std::string &m);  // capi.cu
}
