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
    int32_t family;         /* 0 lane-group kernel, 1 thread-per-run kernel, 2 thread-per-run with
                               the network in global memory (batch kernel, one job), 3 importance
                               sampling (one warp per run), 4 class-coded thread-per-run kernel,
                               5 importance sampling (one thread per run, tilt groups) */
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

/* As csmc_run, from a host blob to host outputs: the blob is copied to the
 * device, the runs simulated, and the per-run outputs copied back into the
 * host buffers (any may be NULL) on every call.  out->sum and out->sum_sq
 * are summed on the host in run order (the reference's host reduction).
 * The library keeps, per device, the network handle of the last blob (its
 * launch plan is reused while the bytes stay the same), device output
 * buffers, pinned staging buffers and a stream; calls on one device are
 * serialised. */
int csmc_run_host(const void *blob, size_t bytes, const csmc_query *q, uint64_t seed, uint64_t first_run,
                  uint64_t n_runs, uint8_t *flags, double *values, uint32_t *steps, csmc_result *out);

/* Frees what csmc_run_host keeps per device (no counterpart in the
 * reference). */
void csmc_run_host_release(void);

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

/* csmc_smc with a full query (double threshold and horizon) and, beyond the
 * reference's report, optional outputs (no counterpart in the reference):
 * json_path (may be NULL) receives a JSON summary with the estimate, its 95%
 * confidence interval (normal approximation) and the Chernoff-Hoeffding
 * epsilon at delta = 0.05; runs_path (may be NULL) a CSV of every run's
 * flag and tracked value. */
int csmc_smc_ex(const char *model_path, int seed, int sims, const csmc_query *q, const char *loc_query,
                const char *json_path, const char *runs_path);

/* Reads an UPPAAL query formula as the reference's model files write them
 * (no counterpart in the reference, which takes the query from its command
 * line): Pr[<=T](<> Template.location), Pr[<=T](<> var OP k) with OP one of
 * >= > <= <, an optional run count Pr[<=T; N], and E[<=T; N](max: var) /
 * E[<=T; N](min: var).  Variables are named as declared (template locals as
 * Template.name).  Fills *q (max_steps 0), the location name for location
 * queries (loc_query, capacity loc_cap; "" otherwise) and *sims (the
 * formula's run count, 0 when absent). */
int csmc_query_parse(const char *xml_path, const char *formula, csmc_query *q, char *loc_query, size_t loc_cap,
                     uint64_t *sims);

/* Sizes a launch would use for this network: lanes per run, components per
 * lane, runs per CTA. */
int csmc_plan(const csmc_net *net, int32_t *lanes_per_run, int32_t *comps_per_lane, int32_t *runs_per_cta);

/* Overrides the launch plan of a network handle (used by the autotuner):
 * family 0 = lane groups of lanes_per_run lanes (power of two <= 32) with
 * comps_per_lane components each; family 2 = one thread per run with the
 * network and run state in global memory (networks larger than shared
 * memory); family 1 = one thread per run; family 4 = one thread per run with
 * class-coded locations (networks with race classes, at most 256 components
 * and 32 locations per automaton; the default for them).  For families 1, 2
 * and 4 lanes and comps_per_lane are ignored.  threads_per_cta: CTA size.
 * Every family gives the same per-run results. */
int csmc_set_plan(csmc_net *net, int32_t family, int32_t lanes_per_run, int32_t comps_per_lane,
                  int32_t threads_per_cta);

/* Autotuner for one network (no counterpart in the reference, which has one
 * fixed launch shape: one CTA per run, one thread per component).  Times
 * csmc_run on runs 0 .. probe_runs-1 for every feasible plan — one thread
 * per run at 64 and 128 threads per CTA, lane groups at 128 and 256 threads
 * per CTA, and the global-memory plan at 64 and 128 — keeps the fastest on
 * the handle and reports it in best (family, lanes_per_run, comps_per_lane,
 * runs_per_cta, kernel_ms of its probe). */
int csmc_autotune(csmc_net *net, const csmc_query *q, uint64_t seed, uint64_t probe_runs, csmc_result *best);

/* ---- Batches: many (network, query) jobs in one persistent launch --------
 * No counterpart in the reference, which simulates one model per process.
 * Job j simulates the runs csmc_run(nets[j], &qs[j], seeds[j], first_runs[j],
 * n_runs[j], ...) would simulate, with the same per-run results; all jobs'
 * runs are drained from one device work queue by one persistent kernel, so
 * small jobs and long runs do not leave the GPU idle the way a sequence of
 * per-network launches does. */
typedef struct csmc_batch csmc_batch;

/* Builds a batch of n_jobs (1 .. 256) jobs on the current device.  first_runs
 * may be NULL (all 0).  The network handles must outlive the batch.  verify
 * != 0 also keeps per-run trace digests and final states (csmc_run_verify's
 * outputs).  Allocates the per-run outputs, the job table, the run-state
 * slabs and pinned host result buffers. */
int csmc_batch_create(csmc_net *const *nets, const csmc_query *qs, const uint64_t *seeds, const uint64_t *first_runs,
                      const uint64_t *n_runs, int32_t n_jobs, int32_t verify, csmc_batch **out);

/* Launch geometry: threads per CTA (32..128, multiple of 32) and CTAs per SM
 * (0: as many as fit). */
int csmc_batch_set_plan(csmc_batch *b, int32_t threads_per_cta, int32_t ctas_per_sm);
int csmc_batch_plan(const csmc_batch *b, int32_t *threads_per_cta, int32_t *ctas_per_sm);

/* Jobs whose networks have min_comps .. 512 components are simulated one
 * warp per run (32 lanes, up to 16 components each) instead of one thread
 * per run; every warp takes those runs first, then joins the one-thread-per-
 * run queue.  0: every job runs one thread per run.  Default 128.  The
 * per-run results do not depend on it.  csmc_batch_group_comps reports the
 * threshold and how many jobs it selects. */
int csmc_batch_set_group_comps(csmc_batch *b, int32_t min_comps);
int csmc_batch_group_comps(const csmc_batch *b, int32_t *min_comps, int32_t *group_jobs);

/* Enqueues the whole batch on stream — counter reset, the simulation, the
 * per-job value sums and the copies of the counters and sums into the
 * batch's pinned host buffers — without allocating or synchronising, so the
 * sequence can be captured into a CUDA graph.  Read the results with
 * csmc_batch_results after the stream has completed. */
int csmc_batch_launch(csmc_batch *b, void *stream);

/* Runs the batch and fills outs[0 .. n_jobs) in csmc_batch_create's job
 * order.  use_graph != 0: the launch sequence is captured once into a CUDA
 * graph (on a private stream) and the graph is replayed on stream.
 * kernel_ms of every result is the device time of the whole batch. */
int csmc_batch_run(csmc_batch *b, int32_t use_graph, void *stream, csmc_result *outs);

/* Results of the last completed launch. */
int csmc_batch_results(const csmc_batch *b, csmc_result *outs);

/* Device per-run outputs of job j (run i of the job at index i; digests and
 * final_state are NULL unless the batch verifies). */
int csmc_batch_outputs(const csmc_batch *b, int32_t job, uint8_t **flags, double **values, uint32_t **steps,
                       uint64_t **digests, uint32_t **final_state);

/* The same outputs copied into host buffers (any may be NULL; synchronous). */
int csmc_batch_outputs_host(const csmc_batch *b, int32_t job, uint8_t *flags, double *values, uint32_t *steps,
                            uint64_t *digests, uint32_t *final_state);

/* Autotuner for the batch: runs a probe batch (each job's runs scaled by
 * probe_fraction, at least one run, every run capped at 2000 race steps) at
 * each candidate geometry (64 and 128 threads per CTA, every CTAs-per-SM
 * count that fits), keeps the fastest, then at that geometry tries the
 * warp-per-run thresholds 0, 64, 128 and 256 components
 * (csmc_batch_set_group_comps) and keeps the fastest; it orders the jobs of
 * each run space by measured cost per run (where no probe run reached the
 * cap), most expensive first, so that the cheapest runs fill the end of the
 * batch. */
int csmc_batch_autotune(csmc_batch *b, double probe_fraction, int32_t *threads_per_cta, int32_t *ctas_per_sm);

void csmc_batch_free(csmc_batch *b);

/* ---- Importance sampling with a learned proposal ------------------------
 * No counterpart in the reference.  The proposal network (16 -> 64 -> 64 ->
 * 1, GELU, BF16 weights) tilts every exponential rate by exp(theta); the
 * parameter block layout is csmc::MlpParams of cusmc_b200/csrc/include/
 * csmc_mlp.h (CSMC_MLP_PARAM_BYTES bytes). */
#define CSMC_MLP_PARAM_BYTES 11024

/* How runs under the proposal evaluate theta (default 0): 0 = CUDA cores in
 * the CPU oracle's operation order (bit-identical runs); 1 = warp-level BF16
 * tensor-core MMAs with FP32 accumulation.  A run is one warp and a step
 * evaluates four feature rows, too few to keep an MMA tile busy, so the
 * CUDA-core evaluation is the faster one.  Weights and estimates are exact
 * for the theta a run used either way. */
int csmc_is_set_inference(csmc_net *net, int32_t tensor_cores);

/* Which kernel simulates runs under the proposal (csmc_is_run; replay
 * always runs one warp per run).  0 (default): one thread per run (result
 * family 5) when the network has race classes (at most 256 components, 32
 * locations per automaton), theta is evaluated on CUDA cores, the state
 * fits and the launch has at least 48 runs per SM (128 when some location
 * of the network is outside the tilt groups; fewer runs finish sooner one
 * warp per run), else one warp per run (family 3); 3: always one
 * warp per run; 5: one thread per run whenever the network qualifies.  The
 * runs, paths and log-likelihood ratios are the same bits either way. */
int csmc_is_set_kernel(csmc_net *net, int32_t family);

/* Where the proposal's features come from for this network (default:
 * count_vars = variables 0..3, scales = 1 / components, no clock):
 * count_vars[4] (variable ids, -1 unused) feed features 5..8 as value *
 * scales[i]; clock_var (-1: none) feeds feature 4 as its value / T, rounded
 * down to a multiple of 1/64.  NULL arrays keep the default for that part;
 * all three defaults restore the default source.  The epidemic's default
 * (its S, E, I, R counts over N) is the first form. */
int csmc_is_set_features(csmc_net *net, const int32_t *count_vars, const float *scales, int32_t clock_var);

/* Runs first_run .. first_run+n_runs-1 under the proposal.  Per-run device
 * outputs (may be NULL): flags, logw (log-likelihood ratio nominal/proposal,
 * FP64), values (tracked max/min), steps.  out->sum / sum_sq are the sums of
 * flag * exp(logw) and of its square; out->estimate = sum / n_runs is the
 * unbiased importance-sampling estimate of the query's probability. */
int csmc_is_run(csmc_net *net, const csmc_query *q, const void *params, uint64_t seed, uint64_t first_run,
                uint64_t n_runs, uint8_t *flags, double *logw, double *values, uint32_t *steps, csmc_result *out,
                void *stream);

/* Replays runs first_run + runs[i] (device list of n_list offsets) under the
 * proposal and writes their CE training rows (csmc::MlpRow, 40 bytes: BF16
 * features, a, b) to rows: four rows per step starting at row_offset[i]
 * (device), weighted by weights[i] (device).  rows holds rows_cap rows; a
 * row that would land at or beyond rows_cap is not written and the call
 * returns CSMC_ERR_LIMIT (offsets that do not match the runs' step counts
 * under the same proposal and inference mode). */
int csmc_is_trace(csmc_net *net, const csmc_query *q, const void *params, uint64_t seed, uint64_t first_run,
                  const uint64_t *runs, const float *weights, const uint64_t *row_offset, uint64_t n_list, void *rows,
                  uint64_t rows_cap, void *stream);

/* Tensor-core (tcgen05) forward pass of the proposal network over n_rows
 * device rows (csmc::MlpRow): theta (device, n_rows floats, clipped). */
int csmc_mlp_forward(const void *params, const void *rows, uint64_t n_rows, float *theta, void *stream);

/* Tensor-core gradient of J = sum over rows of (b theta - a e^theta) with
 * respect to the parameters (host floats, CSMC_MLP_GRAD_FLOATS of them:
 * w1[64][16], b1[64], w2[64][64], b2[64], w3[64], b3); *objective = J.
 * BF16 operands, FP32 accumulation in tensor memory; the per-CTA partial
 * sums are reduced on the device.  The two tensor-core entry points keep a
 * small set of device buffers per device for the life of the process and
 * serialise calls on the same device. */
#define CSMC_MLP_GRAD_FLOATS 5313
int csmc_mlp_grad(const void *params, const void *rows, uint64_t n_rows, float *grad, double *objective,
                  void *stream);

/* `steps` Adam ascent steps on J over n_rows device rows, on the device with
 * one synchronisation at the end.  x (the FP32 master vector in the
 * gradient's layout), m and v (the moments) are host arrays of
 * CSMC_MLP_GRAD_FLOATS entries and *t the step count, all updated in place.
 * Each step packs x into the BF16 parameter block, takes csmc_mlp_grad's
 * gradient g and applies, in IEEE double rounded to nearest, t += 1,
 * m = 0.9 m + 0.1 g, v = 0.999 v + 0.001 g g (the coefficients as
 * 1 - 0.9 and 1 - 0.999 in double), x += lr (m / c1) / (sqrt(v / c2) +
 * 1e-8) with c1 = 1 - 0.9^t and c2 = 1 - 0.999^t from the host's pow,
 * x rounded to FP32.  *j_first and *j_last: J at the first and the last
 * step's parameters (before their update). */
int csmc_mlp_adam(const void *rows, uint64_t n_rows, int32_t steps, double lr, float *x, double *m, double *v,
                  int32_t *t, double *j_first, double *j_last, void *stream);

/* Merges replayed training rows (device buffers): rows of one listed run and
 * one location class (rows row_offset[i] + l, + 4, ..., up to the next
 * run's first row or n_rows) whose features are equal on consecutive steps
 * are summed into one row (a and b added in FP64 in step order, rounded to
 * FP32), and rows whose a and b are both zero are dropped.  J and its
 * gradient are unchanged in exact arithmetic (J is linear in a and b for a
 * fixed feature row).  out (device, room for n_rows rows) receives the
 * merged rows, ordered by run, class and first step; *n_out their count. */
int csmc_mlp_rows_merge(const void *rows, const uint64_t *row_offset, uint64_t n_list, uint64_t n_rows, void *out,
                        uint64_t *n_out, void *stream);

/* ---- Cross-entropy training of the proposal ---------------------------
 * No counterpart in the reference.  The reference's entry point for a run
 * of the statistical model checker is smc() (smc.cuh:14, smc.cu:283-491);
 * these entry points sit beside it for the learned importance-sampling
 * method, so C/C++ hosts and the CLI (--csmc-is) can train without Python.
 *
 * Parameters cross the ABI as the FP32 master vector of CSMC_MLP_GRAD_FLOATS
 * floats: w1[64][16], b1[64], w2[64][64], b2[64], w3[64], b3. */
typedef struct {
    int32_t rounds;          /* maximum CE rounds (>= 1) */
    int32_t adam_steps;      /* Adam steps per round (>= 1), on the round's rows */
    uint64_t runs_per_round; /* runs simulated under the proposal per round */
    uint64_t max_rows;       /* cap on a round's training rows (4 per step of an elite run) */
    double rho;              /* elite fraction, in (0, 1) */
    double lr;               /* Adam step size (beta1 0.9, beta2 0.999, eps 1e-8) */
    int32_t settle;          /* stop after this many consecutive rounds whose level was the goal (0: never) */
    int32_t pad;
} csmc_ce_config;

typedef struct {
    int32_t round;           /* 0-based */
    int32_t elite;           /* elite runs replayed */
    uint64_t rows;           /* training rows */
    double level;            /* the round's level (the goal once at_goal) */
    double j_start, j_end;   /* CE objective before the first and after the last Adam step */
    double estimate;         /* the round's importance-sampling estimate */
    uint64_t hits, capped;   /* runs at the goal; runs stopped by max_steps */
    double mean_steps;       /* race steps per run */
    double kernel_ms;        /* simulation kernel time of the round's runs */
    double run_s, trace_s, adam_s; /* host seconds: runs + selection, replay, Adam steps */
    int32_t at_goal;         /* 1 when the level was the goal */
    int32_t pad;
} csmc_ce_round;

/* Multi-level CE selection of one round (host only).  score = value (max
 * query) or -value (min query); goal = threshold (or -threshold).  The level
 * is min(goal + 1e-9, q), q the (1 - rho)-quantile of the scores with linear
 * interpolation between order statistics (sorted[lo] + (sorted[lo+1] -
 * sorted[lo]) * (h - lo), h = (n - 1)(1 - rho)).  Elite: runs with score >=
 * level, or score > goal once the level is the goal; if none, the
 * max(1, floor(rho n)) highest-scoring runs.  Weights exp(logw - max logw),
 * normalised; runs are kept heaviest first while their rows (4 per step)
 * total at most max_rows (at least one run), and the kept weights are
 * normalised again.  Outputs (capacity n each): elite run indices,
 * weights (float), row_offset (exclusive prefix sums of 4 * steps, in the
 * kept order); *n_elite, *n_rows, *level (in value units) and *at_goal. */
int csmc_ce_select(const double *values, const double *logw, const uint32_t *steps, uint64_t n, double threshold,
                   int32_t is_max, double rho, uint64_t max_rows, uint64_t *elite, float *weights,
                   uint64_t *row_offset, uint64_t *n_elite, uint64_t *n_rows, double *level, int32_t *at_goal);

/* FP32 master vector -> the CSMC_MLP_PARAM_BYTES parameter block (BF16
 * weight matrices, round to nearest even). */
int csmc_mlp_pack(const float *master, void *params);

/* Initial master vector: w1 ~ N(0, 2/10) on the 10 used inputs, w2 ~
 * N(0, 2/64) (Box-Muller over Philox4x32-10 draws keyed by seed), biases and
 * the output layer 0, so theta = 0 (the proposal starts as the nominal model). */
int csmc_mlp_init(uint64_t seed, float *master);

/* CE training on the GPU: per round, runs_per_round runs under the current
 * proposal (runs (k + 1) * 10^7 .. of the stream for round k), the elite
 * selection above, their replay into rows and adam_steps Adam ascents of
 * J = sum (b theta - a e^theta) with the tensor-core gradient.  init and
 * trained are master vectors; params_out (may be NULL) receives the packed
 * trained parameters; log (may be NULL, log_cap entries) one entry per
 * round; *rounds_done the rounds run.  Needs a variable query. */
int csmc_is_train(csmc_net *net, const csmc_query *q, uint64_t seed, const csmc_ce_config *cfg, const float *init,
                  float *trained, void *params_out, csmc_ce_round *log, int32_t log_cap, int32_t *rounds_done);

/* smc() (smc.cuh:14, smc.cu:283-491) with the learned importance-sampling
 * estimate of a variable probability query (IS_ESTIMATE = 0): the settings
 * report, CE training from csmc_mlp_init(seed) with cfg, then sims weighted
 * runs; prints "Result:" with the estimate, its 95% confidence interval and
 * the timing lines, and writes json_path (may be NULL) with the same.  This
 * is the CLI's --csmc-is. */
int csmc_smc_is(const char *model_path, int seed, int sims, const csmc_query *q, const csmc_ce_config *cfg,
                const char *json_path);

/* ---- Numeric primitives ----------------------------------------------------
 * No counterpart in the reference, whose random stream is curand XORWOW
 * (simulation/simulation.cu:756-760) and whose logarithm is the hardware
 * __log2f (simulation.cu:529).  These are the functions whose exact bits
 * define a run here; csmc_numeric_eval evaluates the device code of one of
 * them over n elements of DEVICE arrays a (and b), writing out, and
 * synchronises the stream.  Codes and operands:
 *   CSMC_NUM_PHILOX        a: u32 counters[4n], b: u32 keys[2n] -> u32[4n]
 *                          (Philox4x32-10, Salmon et al., SC'11)
 *   CSMC_NUM_EXP_DELAY     a: u32 draws[n], b: f32 1/rate[n] -> f32 delay
 *                          (-log2(u) / rate, u = ((x >> 8) + 1) 2^-24)
 *   CSMC_NUM_LOG2_F32      a: f32[n] positive normal -> f32 log2
 *   CSMC_NUM_LOG2_F64      a: f64[n] -> f64 log2
 *   CSMC_NUM_EXP2_F64      a: f64[n] -> f64 2^a
 *   CSMC_NUM_POW_F64       a, b: f64[n] -> f64 a^b (the model language's '^')
 *   CSMC_NUM_EXP2_F32      a: f32[n] -> f32 2^a (proposal network)
 *   CSMC_NUM_GELU_F32      a: f32[n] -> f32 GELU (tanh form)
 *   CSMC_NUM_GELU_GRAD_F32 a: f32[n] -> f32 GELU'
 *   CSMC_NUM_PHILOX_STEP   as CSMC_NUM_PHILOX, through the per-step
 *                          factorisation the simulation kernels use
 *                          (counter = step, component group, run low, run high) */
#define CSMC_NUM_PHILOX 0
#define CSMC_NUM_EXP_DELAY 1
#define CSMC_NUM_LOG2_F32 2
#define CSMC_NUM_LOG2_F64 3
#define CSMC_NUM_EXP2_F64 4
#define CSMC_NUM_POW_F64 5
#define CSMC_NUM_EXP2_F32 6
#define CSMC_NUM_GELU_F32 7
#define CSMC_NUM_GELU_GRAD_F32 8
#define CSMC_NUM_PHILOX_STEP 9
int csmc_numeric_eval(int32_t fn, const void *a, const void *b, uint64_t n, void *out, void *stream);

/* Measures the shared-memory bandwidth of the current device (no
 * counterpart in the reference): a kernel on every SM streams conflict-free
 * 16-byte shared-memory loads (about 5 GB per launch, best of three timed
 * launches after one warm-up).  *gbs receives GB/s over the whole device;
 * *sm_mhz (may be NULL) the mean SM clock during the timed launches, from
 * clock64() against %globaltimer.  This is the peak the shared-memory
 * roofline of the thread-per-run simulation kernel is quoted against. */
int csmc_measure_smem_bandwidth(double *gbs, double *sm_mhz);

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
 * (cudaGetSymbolAddress) with that device current, and keeps it with the id
 * of the current context; a later call from another context on that device
 * (after cudaDeviceReset, or from a non-primary context) looks it up again.
 * Make the first call in a context before any stream capture.  Every call on a device shares the one array
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
