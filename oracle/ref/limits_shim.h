/*
 * Force-included (nvcc/g++ -include) into every translation unit of the
 * reference cuSMC build made by oracle/ref/Makefile.  It is test
 * infrastructure: it lets the reference sources compile in place, unmodified,
 * with two fixed limits raised.
 *
 * The reference keeps its compile-time limits in main.cuh (main.cuh:12-31):
 * MAX_VARIABLES (=3) sizes the per-run variable array in shared memory and
 * MAX_EDGES_PER_NODE (=2) sizes the per-component enabled-edge list
 * (simulation/state/shared_run_state.cuh:21,37).  Networks with more variables
 * or more simultaneously enabled edges overflow those arrays.  Defining the
 * header's include guard first makes the reference's main.cuh expand to
 * nothing, so this file supplies the same declarations (the three plain
 * structs and the CLI helper prototype of main.cuh:33-60, which must keep the
 * same layout because main.cu and smc.cu use them) with the two limits taken
 * from -DCSMC_REF_MAX_VARIABLES / -DCSMC_REF_MAX_EDGES.  All debug-print
 * switches stay 0 and SYNC_SIDE_EFFECT stays true, as in the reference.
 */
#pragma once
#define MAIN_CUH 1

#include <cstdint>
#include <iostream>
#include <string>

#ifndef CSMC_REF_MAX_VARIABLES
#define CSMC_REF_MAX_VARIABLES 3
#endif
#ifndef CSMC_REF_MAX_EDGES
#define CSMC_REF_MAX_EDGES 2
#endif

#define VERBOSE 0
#define EXPR_VERBOSE 0
#define REDUCTION_VERBOSE 0
#define EXPR_VERBOSE_EXTRA 0
#define DELAY_VERBOSE 0
#define CHANNEL_VERBOSE 0
#define PRINT_TRANSITIONS 0
#define PRINT_TRANS_ALOHA 0
#define PRINT_VARIABLES 0
#define PRINT_UPDATES 0
#define LISTEN_TO -1
#define QUERYSTATS 0
#define MINIMAL_PRINTS 0
#define TIME_BOUND 10.0
#define MAX_VARIABLES CSMC_REF_MAX_VARIABLES
#define SYNC_SIDE_EFFECT true

constexpr int MAX_EDGES_PER_NODE = CSMC_REF_MAX_EDGES;
constexpr int MAX_CHANNELS = 8;
constexpr bool USE_GLOBAL_MEMORY_CURAND = true;

struct configuration {
    std::string filename;
    int curand_seed;
};

struct model_info {
    int MAX_VALUE_STACK_SIZE = 64;
    int runs_per_block = 1;
    uint32_t num_vars;
};

struct statistics_Configuration {
    int simulations;
    int timeBound;
    int variable_threshhold;
    int variable_id;
    bool isMax;
    bool isEstimate;
    std::string loc_query;
    statistics_Configuration()
        : simulations(0), timeBound(0), variable_threshhold(0), variable_id(0),
          isMax(false), isEstimate(false), loc_query("") {}
    statistics_Configuration(int sims, int t, int thr, int vid, bool mx, bool est,
                             const std::string &lq)
        : simulations(sims), timeBound(t), variable_threshhold(thr), variable_id(vid),
          isMax(mx), isEstimate(est), loc_query(lq) {}
};

bool HandleCommandLineArguments(int argc, char **argv, std::string *filename, int *seed,
                                statistics_Configuration *stats);
