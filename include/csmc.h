/*
 * csmc — C ABI of the B200 statistical model checker for networks of
 * stochastic timed automata (drop-in for the simulation path of cuSMC).
 *
 * Conventions: every entry point returns an int status (CSMC_OK = 0, negative
 * CSMC_ERR_* on failure) and never lets a C++ exception cross the boundary;
 * csmc_last_error() returns the calling thread's last message.  The library
 * owns device memory behind handles; callers own host buffers.  Calls are
 * thread-compatible: one host thread per handle at a time.
 *
 * Which reference interface each entry point replaces (paths are within the
 * reference repository AndreasHolt/cuSMC):
 *   csmc_model_compile   automata_parser/abstract_parser.h:16 (parse) +
 *                        network/domain_optimization_visitor.h:54 (optimize) +
 *                        network/pn_compile_visitor.h:18 +
 *                        automata_parser/variable_usage_visitor.h:153 (registry) +
 *                        smc.cu:407-436 (goal by name)
 *   csmc_net_upload      simulation/state/shared_model_state.cuh:219-225
 *                        (init_shared_model_state)
 *   csmc_run             smc.cu:11-281 (run_statistical_model_checking) +
 *                        simulation/simulation.cuh:18-21 (simulation_kernel launch) +
 *                        simulation/statistics.cuh:126-163 (collect results)
 *   csmc_run_host        the same, with host buffers, including the uploads
 *                        and the result copies
 *   csmc_smc             smc.cuh:14 / smc.cu:283-491 (void smc(configuration,
 *                        statistics_Configuration)): prints the same report
 *                        and writes the same timing CSV
 */
#ifndef CSMC_H
#define CSMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CSMC_OK 0
#define CSMC_ERR_ARG (-1)      /* invalid argument */
#define CSMC_ERR_MODEL (-2)    /* model file rejected by the front end */
#define CSMC_ERR_CUDA (-3)     /* CUDA runtime error (message has details) */
#define CSMC_ERR_LIMIT (-4)    /* network or query outside supported limits */
#define CSMC_ERR_NODEVICE (-5) /* no CUDA device: there is no CPU fallback */
#define CSMC_ERR_TIMEOUT (-6)  /* a bounded device wait gave up */

#define CSMC_QUERY_LOCATION 0 /* Pr[<=T](<> goal): run stops at the goal */
#define CSMC_QUERY_VARIABLE 1 /* per-run max or min of one variable */

typedef struct csmc_net csmc_net; /* device-resident packed network */

typedef struct {
    int32_t kind;        /* CSMC_QUERY_LOCATION or CSMC_QUERY_VARIABLE */
    int32_t var_id;      /* tracked variable (-1 for location queries) */
    int32_t is_max;      /* 1: track the maximum, 0: the minimum */
    int32_t is_estimate; /* 1: mean of the tracked values; 0: fraction beyond threshold */
    double threshold;    /* probability queries: value > threshold (max) or < threshold (min) */
    double horizon;      /* time bound T */
    uint64_t max_steps;  /* per-run race-step cap (0: 10^7); capped runs are counted */
} csmc_query;

typedef struct {
    uint64_t runs;       /* runs simulated */
    uint64_t hits;       /* location query: runs that reached the goal;
                            variable query: runs beyond the threshold */
    uint64_t steps;      /* total race steps over all runs */
    uint64_t capped;     /* runs stopped by max_steps */
    double sum;          /* variable query: sum of per-run values (in run order) */
    double sum_sq;       /* variable query: sum of squares */
    double estimate;     /* location: hits/runs; variable: mean or fraction */
    double kernel_ms;    /* device time of the simulation kernel(s) */
    int32_t lanes_per_run;  /* launch plan used: lanes per run (1: one thread per run) */
    int32_t comps_per_lane; /* components per lane */
    int32_t runs_per_cta;   /* runs in flight per CTA */
    int32_t family;         /* 0 lane-group kernel, 1 thread-per-run kernel */
} csmc_result;

/* Thread-local message of the last failure on this thread. */
const char *csmc_last_error(void);

/* Library version string. */
const char *csmc_version(void);

/* Front end: parses a UPPAAL model, runs the reference's passes and packs
 * the network.  loc_query is "Template.Location" (may be ""); loc_mode != 0
 * applies the location-query goal marking by name.  On success *blob points
 * to a library-allocated buffer of *bytes bytes (free with csmc_free). */
int csmc_model_compile(const char *xml_path, const char *loc_query, int loc_mode, void **blob, size_t *bytes);

/* Canonical text dump of the network as the kernel receives it
 * (free with csmc_free). */
int csmc_model_dump(const char *xml_path, const char *loc_query, int loc_mode, char **text);

/* Number of variables / components of a packed network. */
int csmc_blob_info(const void *blob, size_t bytes, uint32_t *n_vars, uint32_t *n_comps, uint32_t *n_locs);

void csmc_free(void *p);

/* Uploads a packed network to the current device.  The caller keeps blob. */
int csmc_net_upload(const void *blob, size_t bytes, csmc_net **out);
void csmc_net_free(csmc_net *net);

/* Simulates runs first_run .. first_run+n_runs-1 of the counter-based
 * stream keyed by seed.  Per-run outputs are DEVICE pointers and may be NULL:
 * flags[i] = 1 when run i reached the goal (location) or is beyond the
 * threshold (variable); values[i] = tracked max/min (variable query);
 * steps[i] = race steps of run i.  out is filled after the stream is
 * synchronised.  stream is a cudaStream_t (NULL: default stream). */
int csmc_run(const csmc_net *net, const csmc_query *q, uint64_t seed, uint64_t first_run, uint64_t n_runs,
             uint8_t *flags, double *values, uint32_t *steps, csmc_result *out, void *stream);

/* As csmc_run, from a host blob to host outputs (upload, run, copy back;
 * all copies included).  Host output pointers may be NULL. */
int csmc_run_host(const void *blob, size_t bytes, const csmc_query *q, uint64_t seed, uint64_t first_run,
                  uint64_t n_runs, uint8_t *flags, double *values, uint32_t *steps, csmc_result *out);

/* Verification variant: also returns, per run, a 64-bit digest of the event
 * sequence (winner, delay bits, chosen edge, update values, receivers) and the
 * final state (locations then variable bits, n_comps + n_vars words per run).
 * Device pointers; any may be NULL. */
int csmc_run_verify(const csmc_net *net, const csmc_query *q, uint64_t seed, uint64_t first_run, uint64_t n_runs,
                    uint8_t *flags, double *values, uint32_t *steps, uint64_t *digests, uint32_t *final_state,
                    csmc_result *out, void *stream);

/* The reference's smc() flow on one model: same stdout report ("Set number of
 * variables to", the settings block, "Result:" or the three location-query
 * lines, "Time taken" lines) and the same ../results5.csv update.  seed is the
 * CLI seed; sims/time_bound/threshold/var_id/is_max/is_estimate/loc_query
 * mean what statistics_Configuration's fields mean (main.cuh:46-58). */
int csmc_smc(const char *model_path, int seed, int sims, int time_bound, int threshold, int var_id, int is_max,
             int is_estimate, const char *loc_query);

/* Sizes a launch would use for this network: lanes per run, components per
 * lane, runs per CTA. */
int csmc_plan(const csmc_net *net, int32_t *lanes_per_run, int32_t *comps_per_lane, int32_t *runs_per_cta);

/* Overrides the launch plan of a network handle (used by the autotuner):
 * family 0 = lane groups of lanes_per_run lanes (power of two <= 32) with
 * comps_per_lane components each; family 1 = one thread per run (lanes and
 * comps_per_lane are ignored).  threads_per_cta: CTA size. */
int csmc_set_plan(csmc_net *net, int32_t family, int32_t lanes_per_run, int32_t comps_per_lane,
                  int32_t threads_per_cta);

/* Scratch bytes per device behind csmc_run_noalloc (held from the first
 * call on a device until the process exits). */
#define CSMC_NOALLOC_SCRATCH_BYTES (2u * 1024u * 1024u)

/* csmc_run_noalloc — has no counterpart in the reference.
 *
 * The thread-per-run simulation of csmc_run for callers that cannot let a
 * library allocate device memory: hosts that reserve all device memory
 * themselves at start-up and forbid later cudaMalloc/cudaFree, loops in which
 * cudaMalloc's implicit device synchronisation is not acceptable, or
 * frameworks whose own allocator must own every buffer.  The caller passes
 * the packed network twice — blob_host (host memory, for the launch plan) and
 * blob_device (the same bytes in device memory, 16-byte aligned) — and the
 * device output buffers; flags/values/steps as in csmc_run, except that
 * values is required for variable queries.  Nothing is allocated: the
 * kernel's scratch (work and result counters, partial sums, and run-state
 * slabs when a network's run state does not fit in shared memory) is a
 * file-scope device array of CSMC_NOALLOC_SCRATCH_BYTES bytes per device.
 * Networks whose run state needs more than that are rejected with
 * CSMC_ERR_LIMIT; fewer CTAs are launched when the slabs would not all fit.
 *
 * The first call on a device looks the array's device address up
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  Every call on a device shares the one array
 * and overwrites what the previous call left there (the counters are cleared
 * at the start of each call): calls whose work overlaps on the GPU, from
 * several host threads or on several streams, race and return wrong counts.
 * kernel_ms is not measured (0).  Results, run for run, are those of
 * csmc_run with the thread-per-run plan. */
int csmc_run_noalloc(const void *blob_host, const void *blob_device, size_t bytes, const csmc_query *q,
                     uint64_t seed, uint64_t first_run, uint64_t n_runs, uint8_t *flags, double *values,
                     uint32_t *steps, csmc_result *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif
