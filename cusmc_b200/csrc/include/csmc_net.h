/*
 * Packed network blob: the read-only structure-of-arrays image of one
 * stochastic-timed-automata network that the simulation kernels stage into
 * shared memory (and that the CPU oracle reads).  It replaces the reference's
 * pointer-linked SharedModelState (simulation/state/shared_model_state.cuh:
 * 45-217): destinations are local location indices instead of node ids found
 * by scanning levels (simulation/simulation.cu:147-168), only the guards and
 * invariants the kernel acts on are stored, and expressions are flat
 * programs instead of 32-byte pointer-linked records.
 *
 * All sections start on 16-byte boundaries; all integers are little endian.
 */
#ifndef CSMC_NET_H
#define CSMC_NET_H

#include <stdint.h>

#define CSMC_NET_MAGIC 0x314e4d43u /* "CMN1" */
#define CSMC_NET_VERSION 1u

/* Expression handle: two tag bits + 30-bit payload. */
#define CSMC_H_LIT 0u  /* payload: index into consts[] */
#define CSMC_H_VAR 1u  /* payload: variable id */
#define CSMC_H_PN 2u   /* payload: start index into code[] (postfix program, reference PN semantics) */
#define CSMC_H_TREE 3u /* payload: start index into code[] (tree-evaluator semantics) */
#define CSMC_H_TAG(h) ((uint32_t)(h) >> 30)
#define CSMC_H_PAYLOAD(h) ((uint32_t)(h)&0x3fffffffu)
#define CSMC_H_MAKE(tag, p) (((uint32_t)(tag) << 30) | ((uint32_t)(p)&0x3fffffffu))

/* Program instructions: one uint64, low 8 bits opcode, bits 8..31 operand a.
 * Every program starts with a CSMC_OP_HDR instruction whose operand holds
 * CSMC_PROG_* flags and the stack depth the program needs. */
enum csmc_opcode {
    CSMC_OP_END = 0,
    CSMC_OP_PUSH_C,  /* a: const index */
    CSMC_OP_PUSH_V,  /* a: variable id */
    /* postfix (PN) operators: read the top entries WITHOUT popping them and
       push the result (simulation/expressions.cu:88-173, stack_top is passed
       by value) */
    CSMC_OP_ADD, CSMC_OP_SUB, CSMC_OP_MUL, CSMC_OP_DIV, CSMC_OP_POW, CSMC_OP_NEG,
    CSMC_OP_SQRT, CSMC_OP_MOD, CSMC_OP_AND, CSMC_OP_OR, CSMC_OP_LE, CSMC_OP_GE,
    CSMC_OP_LT, CSMC_OP_GT, CSMC_OP_EQ, CSMC_OP_NE, CSMC_OP_NOT,
    CSMC_OP_RANDOM, /* pushes 1.0 (unsupported in the reference kernel) */
    CSMC_OP_DUP,    /* conditional record: pushes the top entry again */
    CSMC_OP_ZERO,   /* compiled/pn records: push 0.0 */
    CSMC_OP_SKIP,   /* a: length; pop one; if |v| > 1e-5 jump over a records */
    /* tree-evaluator operators (simulation/expressions.cu:199-307): proper
       pop-two push-one stack discipline */
    CSMC_OP_TADD, CSMC_OP_TSUB, CSMC_OP_TMUL,
    CSMC_OP_TDIV, /* r == 0 -> 0; result == 0 -> DBL_MIN */
    CSMC_OP_HDR,  /* program header: a = flags | depth << 8 */
    CSMC_OP_COUNT
};

/* Program header flags.  WINDOW: the program only ever reads the two top
 * stack entries (postfix programs without skips, trees of depth <= 2), so it
 * can be evaluated with two registers. */
#define CSMC_PROG_WINDOW 1u
/* CHAIN: the program is x1 x2 op or x1 x2 op x3 op (x: PUSH_C / PUSH_V; op:
 * ADD SUB MUL DIV or TADD TSUB TMUL), a left fold of at most two binary
 * operations that kernels evaluate without the interpreter. */
#define CSMC_PROG_CHAIN 2u

#define CSMC_INS(op, a) ((uint64_t)(op) | ((uint64_t)(a) << 8))
#define CSMC_INS_OP(i) ((uint32_t)((i)&0xffu))
#define CSMC_INS_A(i) ((uint32_t)(((i) >> 8) & 0xffffffu))

/* Guard / invariant operators as stored. */
enum csmc_gop { CSMC_G_LE = 0, CSMC_G_LT = 1, CSMC_G_GE = 2, CSMC_G_GT = 3, CSMC_G_EQ = 4, CSMC_G_FALSE = 5 };

/* Location types (reference node::node_types, include/engine/domain.h:140-147). */
enum csmc_loc_type { CSMC_LOC = 0, CSMC_GOAL = 1, CSMC_BRANCH = 2, CSMC_URGENT = 3, CSMC_COMMITTED = 4 };

typedef struct {
    uint32_t magic, version, total_bytes, header_bytes;
    uint32_t n_comps, n_locs, n_edges, n_guards;
    uint32_t n_updates, n_vars, n_consts, n_code;
    uint32_t max_locs_per_comp, max_edges_per_loc, max_stack, n_clocks;
    uint32_t off_comp, off_loc, off_edge, off_guard;
    uint32_t off_update, off_var, off_const, off_code;
    uint32_t n_channels_max, max_inv_per_loc, max_guards_per_edge, max_updates_per_edge;
    uint32_t flags;          /* CSMC_NET_* */
    uint32_t n_rate_prog;    /* distinct non-literal rate expressions */
    uint32_t n_inv_lit;      /* distinct literal rates (pre-inverted) */
    uint32_t off_loc_rate;   /* uint16 per location: rate slot */
    uint32_t off_inv_lit;    /* float per literal rate: 1/rate (inv_rate of csmc_numeric.h) */
    uint32_t off_rate_prog;  /* uint32 expression handle per rate program */
    uint32_t recv_chan_lo;   /* bit c: some location can receive on channel c (c < 32) */
    uint32_t recv_chan_hi;   /* channels 32..63; bit 31 also stands for every channel >= 63 */
    uint32_t off_clock;      /* uint16 id per clock variable (n_clocks entries) */
    uint32_t off_loc_desc;   /* uint64 delay descriptor per location (CSMC_DESC_*) */
    uint32_t n_classes;      /* race classes in use (with CSMC_NET_RACE_CLASSES; 0: not recorded) */
    uint32_t off_loc_inv1;   /* uint32 per location: its one invariant (CSMC_DESC_INV1), or 0 */
} csmc_net_header; /* 160 bytes */

/* Header flags. */
#define CSMC_NET_RATE_TABLE 1u  /* rates resolved through loc_rate (see below) */
#define CSMC_NET_RACE_CLASSES 2u /* delay descriptors carry race classes (see below) */
#define CSMC_NET_RATE_NO_CLOCK 4u /* no rate program reads a clock: the rate table
                                     changes only when a transition writes a variable */

/* Rate slot of a location (loc_rate[]): bit 15 set -> index into the
 * per-step table of evaluated rate programs (rate_prog[]); clear -> index
 * into inv_lit[].  Distinct rate programs are evaluated once per step per
 * run instead of once per component. */
#define CSMC_RATE_PROG_BIT 0x8000u
#define CSMC_MAX_RATE_PROGS 64

/* Delay descriptor of a location (loc_desc[]): everything the per-component
 * delay needs in one 8-byte word.  Low 32 bits: the float 1/rate of a
 * literal rate, or the rate-table slot of a rate program (DESC_PROG).  High
 * 32 bits: flags. */
#define CSMC_DESC_PROG (1u << 0)  /* low word is a rate-table slot */
#define CSMC_DESC_ZERO (1u << 1)  /* branch / urgent / committed: delay 0 */
#define CSMC_DESC_INV (1u << 2)   /* has delay-bounding invariants */
#define CSMC_DESC_EVAL (1u << 3)  /* rate evaluated per component (no table) */
/* INV1 (with INV): the location's only delay-bounding invariant is clock var
 * < or <= a literal; loc_inv1[] holds var << 16 | strict << 15 | the
 * literal's const index (< 2^15).  Never set together with EVAL. */
#define CSMC_DESC_INV1 (1u << 4)
#define CSMC_INV1_VAR(w) ((w) >> 16)
#define CSMC_INV1_STRICT(w) (((w) >> 15) & 1u)
#define CSMC_INV1_CONST(w) ((w)&0x7fffu)
/* Race class (high word bits 8..15; 0xff: none): locations whose delay is
 * always exponential with 1/rate from the same literal or the same per-step
 * rate program.  Within a class the delay is a non-increasing function of
 * the 24-bit uniform draw, so the race only needs each class's largest draws
 * (set, with CSMC_NET_RACE_CLASSES, when a network has at most
 * CSMC_RACE_CLASSES classes and at most 256 components). */
#define CSMC_DESC_CLASS(fl) (((fl) >> 8) & 0xffu)
#define CSMC_DESC_NO_CLASS 0xffu
#define CSMC_RACE_CLASSES 4

typedef struct {
    uint32_t loc_begin;  /* global index of the component's first location */
    uint16_t n_locs;
    uint16_t init_local; /* initial location, local index */
} csmc_comp;             /* 8 bytes */

typedef struct {
    uint32_t edge_begin;
    uint32_t inv_begin;  /* into guards[]: delay-bounding invariants only */
    uint32_t rate;       /* expression handle of the exponential rate */
    uint8_t type;        /* csmc_loc_type */
    uint8_t n_edges;
    uint8_t n_inv;
    uint8_t n_recv;      /* number of receiving edges (channel < 0) */
} csmc_loc;              /* 16 bytes */

typedef struct {
    int16_t dst_local;   /* -1: destination not in this component (no move) */
    int16_t channel;     /* 0 tau, >0 broadcast sender, <0 receiver */
    uint32_t weight;      /* expression handle (tree semantics) */
    uint32_t guard_begin; /* guard_begin (24 bits) | n_guards << 24 */
    uint32_t upd;         /* update_begin (24 bits) | n_updates << 24 */
} csmc_edge; /* 16 bytes */

#define CSMC_EDGE_GUARD_BEGIN(e) ((e).guard_begin & 0xffffffu)
#define CSMC_EDGE_N_GUARDS(e) ((e).guard_begin >> 24)
#define CSMC_EDGE_UPD_BEGIN(e) ((e).upd & 0xffffffu)
#define CSMC_EDGE_N_UPD(e) ((e).upd >> 24)

typedef struct {
    uint16_t var;
    uint8_t op;    /* csmc_gop */
    uint8_t clock; /* 1 when var is a clock */
    uint32_t rhs;  /* expression handle */
} csmc_guard;      /* 8 bytes */

typedef struct {
    uint32_t var;
    uint32_t expr; /* expression handle (PN semantics) */
} csmc_update;     /* 8 bytes */

typedef struct {
    float init;    /* initial value (int-truncated, as the reference uploads it) */
    uint32_t kind; /* 1 clock, 0 int */
} csmc_var;        /* 8 bytes */

/* Limits of the packed form. */
#define CSMC_MAX_EDGES_PER_LOC 32 /* enabled-edge slot state is a 32-bit mask */
#define CSMC_MAX_STACK 32         /* expression stack entries */

#endif
