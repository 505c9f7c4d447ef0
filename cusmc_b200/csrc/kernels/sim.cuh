// Simulation kernel for sm_100a: the reference's per-run loop
// (simulation/simulation.cu:674-901) re-mapped onto lane groups.
//
// Mapping.  One run is simulated by a group of G lanes (G a power of two,
// G <= 32); lane l of a group owns components l*K .. l*K+K-1.  Several groups
// share a warp when G < 32.  The packed network (read-only, a few KB to a few
// hundred KB) is staged once per CTA into shared memory; each group keeps its
// run's variables, broadcast channel, goal flag and query extrema in shared
// memory, and each lane keeps its components' locations and enabled-edge slot
// masks in registers.  There are no block-wide barriers in the loop: a step is
//   1. broadcast receivers of the previous step's sender (enabled sets in
//      parallel, transitions serially in component order);
//   2. per-component delays (lane-parallel);
//   3. the race: a segmented xor-butterfly min over (delay key, bit-reversed
//      component index), which reproduces the reference's strided
//      shared-memory tree argmin (simulation/simulation.cu:576-628) exactly,
//      ties included;
//   4. clock advance (lane-parallel over variables) and the winner's
//      transition (one lane).
// Runs are pulled from a device work counter, so groups whose runs end early
// refill immediately (persistent kernel, grid = resident CTAs).
#pragma once
#include <cstdint>

#include "../include/csmc_net.h"
#include "../include/csmc_numeric.h"
#include "../include/csmc_mlp.h"

// Tilt groups of the thread-per-run importance-sampling kernel: 3-bit
// location codes 0..5 (6 pads the last location word, 7 is the descriptor
// path).
#define CSMC_IS_GROUPS 6

namespace csmc {

// Section offsets and counts of the packed network (copied from its header
// by the host, so kernels read them from the parameter bank).
struct NetLayout {
    uint32_t off_comp, off_loc, off_edge, off_guard, off_update, off_var, off_const, off_code;
    uint32_t off_loc_rate, off_inv_lit, off_rate_prog, off_clock, off_loc_desc;
    uint32_t n_comps, n_vars, n_rate_prog, flags, n_clocks, recv_lo, recv_hi;
    uint32_t n_classes;  // race classes in use (CSMC_RACE_CLASSES when the blob does not record it)
    uint32_t off_loc_inv1;  // one-invariant table (0: none)
};

inline NetLayout layout_of(const csmc_net_header &h) {
    const uint32_t ncls = (h.n_classes && h.n_classes <= CSMC_RACE_CLASSES) ? h.n_classes : CSMC_RACE_CLASSES;
    return NetLayout{h.off_comp,     h.off_loc,     h.off_edge,      h.off_guard,    h.off_update,
                     h.off_var,      h.off_const,   h.off_code,      h.off_loc_rate, h.off_inv_lit,
                     h.off_rate_prog, h.off_clock,  h.off_loc_desc,  h.n_comps,      h.n_vars,
                     h.n_rate_prog,  h.flags,       h.n_clocks,      h.recv_chan_lo, h.recv_chan_hi,
                     ncls,           h.off_loc_inv1};
}

struct SimParams {
    NetLayout net;             // layout of the network staged at the start of shared memory
    const uint8_t *blob;       // packed network in global memory
    uint32_t blob_bytes;       // bytes to stage (multiple of 16)
    uint32_t state_stride;     // bytes of per-group run state in shared memory (multiple of 16)
    int32_t loc_mode;          // CSMC_QUERY_LOCATION
    int32_t var_id;            // tracked variable or -1
    int32_t is_max;
    int32_t pad0;
    double threshold;
    float horizon;             // time bound as the reference's float time_bound
    uint32_t pad1;
    uint64_t max_steps;
    uint64_t seed;
    uint64_t first_run;
    uint64_t n_runs;
    uint8_t *flags;            // per-run outputs (may be null)
    double *values;
    uint32_t *steps;
    uint64_t *digests;         // verification outputs (may be null)
    uint32_t *final_state;
    unsigned long long *scratch;  // [0] work counter [1] hits [2] steps [3] capped [4] errors
    uint8_t *state_global;        // thread-per-run kernel: per-CTA state slabs in global memory
                                  // (null: state in shared memory after the network)
    PhiloxKeys keys;              // round keys of the seed (philox_keys(seed)): read from the
                                  // parameter bank by the class-coded kernel
    uint32_t class_src[CSMC_RACE_CLASSES];  // class-coded kernel: each race class's 1/rate,
                                  // CSMC_CLASS_SRC_PROG | rate-table slot, or the literal's float bits
};
#define CSMC_CLASS_SRC_PROG 0x80000000u

#define CSMC_SCRATCH_WORDS 8

// Launch entry points (sim_dispatch.cu).  Lane-group kernel family:
int sim_launch(int lanes_per_run, int comps_per_lane, bool verify, const SimParams &p, int grid, int block,
               size_t smem, void *stream);
int sim_max_active_ctas(int lanes_per_run, int comps_per_lane, bool verify, int block, size_t smem, int *ctas);
bool sim_supported(int lanes_per_run, int comps_per_lane);
// Thread-per-run kernel family (slots: the network has locations with
// several edges, so enabled-edge slot masks are kept):
// loc8: locations kept as 8-bit local indices (every automaton has at most
// 256 locations); gstate: run state in global slabs instead of shared memory.
// classes: the network's delay descriptors carry race classes.
int serial_launch(bool verify, bool slots, bool loc8, bool gstate, bool classes, const SimParams &p, int grid,
                  int block, size_t smem, void *stream);
int serial_max_active_ctas(bool verify, bool slots, bool loc8, bool gstate, bool classes, int block, size_t smem,
                           int *ctas);

// Class-coded thread-per-run kernel (sim_coded.cuh): networks with race
// classes, at most 256 components and at most 32 locations per automaton,
// run state in shared memory.
// all_classed: every location of the network belongs to a race class.
int coded_launch(bool verify, bool slots, bool all_classed, const SimParams &p, int grid, int block, size_t smem,
                 void *stream);
int coded_max_active_ctas(bool verify, bool slots, bool all_classed, int block, size_t smem, int *ctas);
// Bytes of a T-thread state slab of the class-coded kernel
// (carve_coded_view): n_classes race classes, recv: the network has
// receiving edges (the receiver snapshot is kept).
inline size_t coded_slab_bytes(uint32_t n_comps, uint32_t n_vars, uint32_t n_rate_prog, bool slots, uint32_t T,
                               uint32_t n_classes, bool recv) {
    size_t b = 4u * ((recv ? 2u : 1u) * n_vars + n_rate_prog) * static_cast<size_t>(T);
    b += 4u * 4u * n_classes * static_cast<size_t>(T);             // class keys: the largest of each chain
    b += 4u * ((n_comps + 3u) / 4u) * static_cast<size_t>(T);        // location words
    if (slots) b += 4u * n_comps * static_cast<size_t>(T);          // enabled-edge slot masks
    return (b + 15u) & ~static_cast<size_t>(15);
}

// ---- Multi-network batch kernel (sim_batch.cuh) ---------------------------
// One persistent launch simulates the runs of many (network, query) jobs.
// The runs of all jobs form one index space (job j owns [run_begin,
// run_begin + n_runs)); every lane takes its next run from one device
// counter, so a lane moves on to the next job the moment the current one has
// no runs left, whatever the other lanes are doing.  Networks are read from
// global memory (L1/L2-cached), run state lives in per-CTA global slabs laid
// out for the largest job.  Results depend only on (job, run index), not on
// which lane ran it.
struct BatchJob {
    NetLayout net;
    const uint8_t *blob;           // the job's packed network (device, 16-byte aligned)
    uint64_t run_begin;            // first index of the job in the batch's run space
    uint64_t n_runs;
    uint64_t first_run;            // stream index of the job's first run
    uint64_t seed;
    uint64_t max_steps;
    double threshold;
    float horizon;
    int32_t loc_mode, var_id, is_max;
    uint8_t *flags;                // per-run outputs of the job (may be null)
    double *values;
    uint32_t *steps;
    uint64_t *digests;             // verification outputs (may be null)
    uint32_t *final_state;
    unsigned long long *counters;  // [0] hits [1] steps [2] capped
};
static_assert(sizeof(BatchJob) % 16 == 0, "BatchJob is copied in 16-byte words");

// Job table: the n_group_jobs warp-per-run jobs first, then the thread-per-
// run jobs; each part sorted by run_begin within its own run space.
struct BatchParams {
    const BatchJob *jobs;          // device job table
    uint32_t n_jobs;
    uint32_t state_stride;         // bytes of one CTA's thread-per-run state slab
    uint64_t total_runs;           // runs of the thread-per-run jobs
    unsigned long long *queue;     // the thread-per-run jobs' run counter
    uint8_t *state;                // grid * state_stride bytes
    uint32_t max_vars, max_rate_prog, max_comps;  // maxima over the thread-per-run jobs
    uint32_t n_group_jobs;         // jobs simulated one warp per run (0: none)
    uint64_t group_runs;           // runs of the warp-per-run jobs
    unsigned long long *group_queue;  // their run counter (null when n_group_jobs is 0)
    uint32_t group_stride;         // shared memory of one warp's run state (group_state_stride over the jobs)
    uint32_t group_k;              // components per lane of the warp-per-run jobs: 4, 8 or 16
};

#define CSMC_BATCH_MAX_JOBS 256
// Largest network a batch job can run one warp per run: 32 lanes x 16
// components.
#define CSMC_BATCH_GROUP_MAX_COMPS 512

int batch_launch(bool verify, const BatchParams &p, int grid, int block, void *stream);
// group_k: 0 (thread per run only) or the components per lane of the
// warp-per-run jobs (4, 8 or 16)
int batch_max_active_ctas(bool verify, int group_k, int block, size_t smem, int *ctas);
inline size_t batch_smem_bytes(uint32_t n_jobs) { return static_cast<size_t>(n_jobs) * sizeof(BatchJob); }
// Shared memory of a batch launch: the job table, then one warp-per-run
// state per warp when some job runs one warp per run.
inline size_t batch_smem_bytes(uint32_t n_jobs, uint32_t group_stride, int block) {
    return batch_smem_bytes(n_jobs) + (group_stride ? static_cast<size_t>(block / 32) * group_stride : 0);
}
// Shared memory of one lane group's run state (sim_impl.cuh: RunState): 48
// bytes of scalars, the variables and one inverse rate per rate program,
// 16-aligned; then the group's slot masks, component gl*K + k of lane gl at
// [k * lanes + gl].
__host__ __device__ inline uint32_t group_vars_bytes(uint32_t n_vars, uint32_t n_rate_prog) {
    return (48u + 4u * (n_vars + n_rate_prog) + 15u) & ~15u;
}
__host__ __device__ inline uint32_t group_state_stride(uint32_t n_vars, uint32_t n_rate_prog, uint32_t lanes,
                                                       uint32_t comps_per_lane) {
    // 16-aligned: the next group's scalars hold doubles
    return (group_vars_bytes(n_vars, n_rate_prog) + 4u * lanes * comps_per_lane + 15u) & ~15u;
}
// Bytes of one thread's state in a batch slab (16-bit locations, slot masks).
inline size_t batch_state_bytes_per_thread(uint32_t max_comps, uint32_t max_vars, uint32_t max_rate_prog) {
    return 4u * (2u * max_vars + max_rate_prog + 2u * CSMC_RACE_CLASSES) + 2u * max_comps + 4u * max_comps + 4u;
}

// ---- Importance sampling (sim_is.cuh) --------------------------------------
// One warp per run under the proposal network; trace mode replays listed
// runs and writes their CE training rows.
struct IsParams {
    SimParams s;                  // network, query, run range; s.values: tracked values
    const MlpParams *mlp;         // proposal network (device)
    double *logw;                 // per run: log-likelihood ratio (may be null)
    double *wvals;                // per run: flag * exp(logw) (may be null)
    const uint64_t *trace_runs;   // trace mode: run offsets from s.first_run, s.n_runs of them
    const float *trace_w;         // trace mode: CE weight per listed run
    const uint64_t *row_offset;   // trace mode: first row of each listed run (4 rows per step)
    MlpRow *rows;                 // trace mode: the rows
    uint64_t rows_cap;            // trace mode: rows the buffer holds (writes beyond it are skipped, counted)
    uint32_t slab_bytes;          // shared memory of one warp (is_warp_slab_bytes)
    uint32_t n_groups;            // thread-per-run kernel: tilt groups in use (<= CSMC_IS_GROUPS)
    MlpFeatures feat;             // where the proposal's features come from
    // thread-per-run kernel (sim_is_coded.cuh): the tilt groups, i.e. the
    // (race class, location class) pairs of the network's classed
    // locations.  group_map holds, at bits 3 (4 g + l), the 3-bit location
    // code of race class g in location class l: a group index, or 7 (the
    // descriptor path) for pairs beyond the first CSMC_IS_GROUPS.
    uint64_t group_map;
    uint32_t group_l;                       // location class of group i at bits 2i .. 2i + 1
    uint32_t group_src[CSMC_IS_GROUPS];     // 1/rate source of group i (SimParams::class_src format)
    // thread-per-run kernel: device-wide cache of the class factors by
    // feature vector (CSMC_THETA_CACHE_WORDS words per entry, cache_mask + 1
    // entries; null: none); entries of other generations are empty
    uint32_t *theta_cache;
    uint32_t cache_mask;
    uint32_t cache_gen;                     // the parameter block's generation (bit 31 clear, not 0)
};
// Theta cache entry: [0] state (generation, or generation | 1 << 31 while
// being written), [1..3] the feature key, [4..7] the four class factors.
#define CSMC_THETA_CACHE_WORDS 8

// Importance sampling one thread per run (sim_is_coded.cuh), for networks
// with race classes (at most 256 components, 32 locations per automaton):
// the CUDA-core evaluation of theta, no trace mode.  Shared memory: the
// network, the proposal network's FP32 copies, each warp's first-hidden-layer staging,
// then is_coded_slab_bytes of run state.
// all_grouped: every location belongs to a tilt group and the component
// count is a multiple of four (no descriptor path, no padding in the race).
int is_coded_launch(bool slots, bool all_grouped, const IsParams &p, int grid, int block, size_t smem, void *stream);
int is_coded_max_active_ctas(bool slots, bool all_grouped, int block, size_t smem, int *ctas);
// Shared memory of the proposal network in that kernel (the FP32 copies),
// and of one warp's staging of the first hidden layer.
size_t is_coded_mlp_smem_bytes();
size_t is_coded_warp_smem_bytes();
// Run state of a CTA of T threads: per thread and tilt group the step's
// 1/rate, 1/rate' and FP64 rate change (4 words), then the class-coded
// layout with one key chain set per tilt group.
inline size_t is_coded_slab_bytes(uint32_t n_comps, uint32_t n_vars, uint32_t n_rate_prog, bool slots, uint32_t T,
                                  uint32_t n_groups, bool recv) {
    return 16u * n_groups * static_cast<size_t>(T) + coded_slab_bytes(n_comps, n_vars, n_rate_prog, slots, T,
                                                                     n_groups, recv);
}

// tc: theta by warp-level tensor-core MMAs (else the CUDA-core evaluation
// that is bit-identical to the CPU oracle).
int is_launch(bool tc, bool trace, bool slots, bool loc8, const IsParams &p, int grid, int block, size_t smem,
              void *stream);
int is_max_active_ctas(bool tc, bool trace, bool slots, bool loc8, int block, size_t smem, int *ctas);
// Shared memory of the importance-sampling kernel besides the network: the
// proposal network once per CTA, then one slab per warp holding the run's
// state (the thread-per-run layout with one thread) and, for the CUDA-core
// evaluation, the first hidden layer of the step's four rows.
size_t is_mlp_smem_bytes();
#ifndef CSMC_IS_BLOCK
#define CSMC_IS_BLOCK 256  // threads per CTA of the importance-sampling kernel (eight runs)
#endif
inline size_t is_warp_slab_bytes(size_t run_state_bytes, bool tc) {
    return (tc ? 0u : 4u * CSMC_MLP_HID * CSMC_MLP_CLASSES) + ((run_state_bytes + 15u) & ~static_cast<size_t>(15));
}

// Tensor-core kernels of the proposal network (mlp_train.cu): mode 0 writes
// theta per row, mode 1 gradient partials per CTA (mlp_tc_partial_floats()
// floats each) and the objective per CTA.
int mlp_tc_launch(int mode, const MlpRow *rows, uint64_t n_rows, const MlpParams *P, float *theta_out,
                  float *partials, double *objective, int *error, int grid, void *stream);
int mlp_tc_partial_floats();

// Bytes of thread-per-run state per thread for a network.
inline size_t serial_state_bytes_per_thread(uint32_t n_comps, uint32_t n_vars, uint32_t n_rate_prog, bool slots,
                                            bool loc8) {
    size_t b = 4u * (2u * n_vars + n_rate_prog);        // variables, rate table, receiver snapshot
    b += 4u * 2u * CSMC_RACE_CLASSES;                   // race-class keys
    b += loc8 ? ((n_comps + 3u) & ~3u) : ((2u * n_comps + 3u) & ~3u);  // locations
    if (slots) b += 4u * n_comps;                       // enabled-edge slot masks
    return b;
}

}  // namespace csmc
