/*
 * The proposal network of importance sampling, as plain arithmetic shared by
 * the CPU oracle and the CUDA kernels (same operations in the same order,
 * so both give the same bits).
 *
 * Proposal.  In a run simulated under the proposal, every component whose
 * delay is exponential draws it with its rate multiplied by exp(theta),
 * theta = MLP(features) clipped to [-CSMC_MLP_THETA_MAX, CSMC_MLP_THETA_MAX].
 * Uniform (invariant-bounded) and zero delays, edge choices and updates are
 * unchanged.  The run carries the log-likelihood ratio of its path (nominal
 * over proposal) in FP64, so weight * goal indicator is an unbiased estimate
 * of the goal probability.
 *
 * Features of a component (CSMC_MLP_IN = 16 inputs, 10 used), from a
 * per-network feature source (MlpFeatures):
 *   [0..3]  one-hot of its local location index modulo 4
 *   [4]     the value of the network's chosen clock variable / T, rounded
 *           down to a multiple of 1/CSMC_MLP_TIME_STEPS (0 when the network
 *           chooses none; one clock shared by every component, so the
 *           components of a location class keep sharing their features)
 *   [5..8]  four chosen variables times their scales (default: variables
 *           0..3 times 1/C, for the epidemic network the S, E, I, R
 *           fractions; 0 for an unused slot)
 *   [9]     time / T rounded down to a multiple of 1/CSMC_MLP_TIME_STEPS
 * rounded to BF16 (the time feature takes 64 values over the horizon, so the
 * network is evaluated again at most 64 times per run because time passed).  All components in the same local location share their
 * features, so a run needs one network evaluation per location class and
 * step.
 *
 * Network: 16 -> 64 (GELU) -> 64 (GELU) -> 1, BF16 weights, FP32
 * accumulation; the first hidden layer's activations are rounded to BF16
 * (the tensor-core training kernels consume them in BF16).  GELU is the tanh
 * form x * sigmoid(2 * sqrt(2/pi) * (x + 0.044715 x^3)) with the exponential
 * evaluated by the project's own exp2 (range reduction to [-1/2, 1/2] and a
 * degree-7 Taylor polynomial of e^(f ln 2)).
 */
#ifndef CSMC_MLP_H
#define CSMC_MLP_H

#include "csmc_numeric.h"

#define CSMC_MLP_IN 16
#define CSMC_MLP_HID 64
#define CSMC_MLP_FEATURES 10
#define CSMC_MLP_THETA_MAX 4.0f
#define CSMC_MLP_CLASSES 4
#define CSMC_MLP_TIME_STEPS 64.0f

namespace csmc {

/* Parameter block (all BF16 bit patterns except where noted), as uploaded:
 *   w1[HID][IN]   layer 1, row = output unit
 *   b1[HID]       FP32
 *   w2[HID][HID]  layer 2, row = output unit
 *   b2[HID]       FP32
 *   w3[HID]       FP32 output weights (applied on CUDA cores)
 *   b3            FP32 */
struct MlpParams {
    uint16_t w1[CSMC_MLP_HID][CSMC_MLP_IN];
    float b1[CSMC_MLP_HID];
    uint16_t w2[CSMC_MLP_HID][CSMC_MLP_HID];
    float b2[CSMC_MLP_HID];
    float w3[CSMC_MLP_HID];
    float b3;
    float pad[3];
};
static_assert(sizeof(MlpParams) == 11024, "parameter block layout (CSMC_MLP_PARAM_BYTES)");

CSMC_HD float bf16_to_f(uint16_t h) { return bits_f(static_cast<uint32_t>(h) << 16); }

/* FP32 -> BF16, round to nearest even (NaN kept quiet). */
CSMC_HD uint16_t f_to_bf16(float x) {
    const uint32_t b = f_bits(x);
    if ((b & 0x7fffffffu) > 0x7f800000u) return static_cast<uint16_t>((b >> 16) | 0x40u);
    const uint32_t r = b + 0x7fffu + ((b >> 16) & 1u);
    return static_cast<uint16_t>(r >> 16);
}

CSMC_HD float bf16_round(float x) { return bf16_to_f(f_to_bf16(x)); }

/* 2^t for t in [-126, 126] (clamped): t = n + f, |f| <= 1/2, 2^f = e^(f ln2)
 * by its Taylor polynomial to degree 7 (relative error below 1e-8). */
CSMC_HD float exp2_f(float t) {
    t = t < -126.0f ? -126.0f : (t > 126.0f ? 126.0f : t);
    const float n = static_cast<float>(static_cast<int>(t >= 0.0f ? f_add(t, 0.5f) : f_add(t, -0.5f)));
    const float g = f_mul(f_add(t, -n), 0.693147182f);
    float p = 1.98412701e-4f;        // 1/5040
    p = f_fma(p, g, 1.38888892e-3f);  // 1/720
    p = f_fma(p, g, 8.33333377e-3f);  // 1/120
    p = f_fma(p, g, 4.16666679e-2f);  // 1/24
    p = f_fma(p, g, 0.166666672f);    // 1/6
    p = f_fma(p, g, 0.5f);
    p = f_fma(p, g, 1.0f);
    p = f_fma(p, g, 1.0f);
    const int e = static_cast<int>(n);
    return f_mul(p, bits_f(static_cast<uint32_t>(e + 127) << 23));
}

/* sigmoid(s) = 1 / (1 + 2^(-s log2 e)) */
CSMC_HD float sigmoid_f(float s) { return f_div(1.0f, f_add(1.0f, exp2_f(f_mul(s, -1.44269502f)))); }

/* GELU, tanh form, and its derivative. */
CSMC_HD float gelu_arg(float x) {
    const float x3 = f_mul(f_mul(x, x), x);
    return f_mul(1.59576912f, f_fma(0.044715f, x3, x));
}
CSMC_HD float gelu_f(float x) { return f_mul(x, sigmoid_f(gelu_arg(x))); }
CSMC_HD float gelu_grad_f(float x) {
    const float s = sigmoid_f(gelu_arg(x));
    const float ds = f_mul(s, f_add(1.0f, -s));                              // sigmoid'
    const float dz = f_mul(1.59576912f, f_fma(f_mul(0.134145f, x), x, 1.0f));  // d(arg)/dx
    return f_fma(f_mul(x, ds), dz, s);
}

/* GELU and its derivative sharing one sigmoid (the same bits as gelu_f and
 * gelu_grad_f). */
CSMC_HD void gelu_both(float x, float &g, float &dg) {
    const float s = sigmoid_f(gelu_arg(x));
    const float ds = f_mul(s, f_add(1.0f, -s));
    const float dz = f_mul(1.59576912f, f_fma(f_mul(0.134145f, x), x, 1.0f));
    g = f_mul(x, s);
    dg = f_fma(f_mul(x, ds), dz, s);
}

/* Where a network's features come from: var[i] >= 0 feeds feature 5 + i as
 * value * scale[i]; clock_var >= 0 feeds feature 4. */
struct MlpFeatures {
    int32_t var[4];
    float scale[4];
    int32_t clock_var;
    int32_t pad[3];
};

/* The default source: variables 0..3 (those that exist) over C components,
 * no clock. */
CSMC_HD MlpFeatures mlp_default_features(uint32_t n_vars, uint32_t C) {
    MlpFeatures F;
    const float inv_c = f_div(1.0f, static_cast<float>(C));
    for (int i = 0; i < 4; ++i) {
        F.var[i] = static_cast<uint32_t>(i) < n_vars ? i : -1;
        F.scale[i] = inv_c;
    }
    F.clock_var = -1;
    F.pad[0] = F.pad[1] = F.pad[2] = 0;
    return F;
}

/* t / T rounded down to a multiple of 1/CSMC_MLP_TIME_STEPS (t >= 0, so
 * the truncation is the floor; the multiples up to 1 are exact in BF16). */
CSMC_HD float mlp_time_feature(float t, float T) {
    const float steps = static_cast<float>(static_cast<int>(f_mul(f_div(t, T), CSMC_MLP_TIME_STEPS)));
    return bf16_round(f_div(steps, CSMC_MLP_TIME_STEPS));
}

/* Features of location class l (local index modulo 4): v[i] the value of
 * F.var[i] (ignored when unused), clk the value of F.clock_var, time t,
 * horizon T; BF16-rounded. */
CSMC_HD void mlp_features(uint32_t l, const MlpFeatures &F, const float *v, float clk, float t, float T, float *x) {
    for (int i = 0; i < CSMC_MLP_IN; ++i) x[i] = 0.0f;
    x[l & 3u] = 1.0f;
    if (F.clock_var >= 0) x[4] = mlp_time_feature(clk, T);
    for (int i = 0; i < 4; ++i)
        if (F.var[i] >= 0) x[5 + i] = bf16_round(f_mul(v[i], F.scale[i]));
    x[9] = mlp_time_feature(t, T);
}

/* Sums in the order of a 32-lane warp.  A run is simulated by one warp:
 * component c belongs to lane (c / 4) mod 32 (the lane that draws its
 * Philox block), each lane sums its own terms in component order, and the
 * lanes' partial sums meet in a butterfly (offsets 16, 8, 4, 2, 1; lane L
 * adds lane L ^ off's value to its own, so every lane ends with the same
 * bits).  The CPU restatement keeps the 32 partial sums in an array. */
#define CSMC_WARP 32
CSMC_HD uint32_t warp_lane_of(uint32_t c) { return (c >> 2) & (CSMC_WARP - 1u); }
static_assert(CSMC_MLP_HID == 2 * CSMC_WARP, "each lane holds two hidden units");

CSMC_HD double warp_tree_d(double *p) {
    for (uint32_t off = CSMC_WARP / 2; off > 0; off >>= 1) {
        double q[CSMC_WARP];
        for (uint32_t l = 0; l < CSMC_WARP; ++l) q[l] = d_add(p[l], p[l ^ off]);
        for (uint32_t l = 0; l < CSMC_WARP; ++l) p[l] = q[l];
    }
    return p[0];
}

CSMC_HD float warp_tree_f(float *p) {
    for (uint32_t off = CSMC_WARP / 2; off > 0; off >>= 1) {
        float q[CSMC_WARP];
        for (uint32_t l = 0; l < CSMC_WARP; ++l) q[l] = f_add(p[l], p[l ^ off]);
        for (uint32_t l = 0; l < CSMC_WARP; ++l) p[l] = q[l];
    }
    return p[0];
}

CSMC_HD float clip_theta(float th) {
    return th < -CSMC_MLP_THETA_MAX ? -CSMC_MLP_THETA_MAX : (th > CSMC_MLP_THETA_MAX ? CSMC_MLP_THETA_MAX : th);
}

/* theta for one feature row: first layer and GELU, activations rounded to
 * BF16, second layer and GELU (each unit's dot product in input order),
 * output layer in warp order (lane L: units L and L + 32, then the
 * butterfly), plus the output bias, clipped. */
CSMC_HD float mlp_theta(const MlpParams &P, const float *x) {
    float h1[CSMC_MLP_HID];
    for (int j = 0; j < CSMC_MLP_HID; ++j) {
        float z = P.b1[j];
        for (int i = 0; i < CSMC_MLP_IN; ++i) z = f_fma(x[i], bf16_to_f(P.w1[j][i]), z);
        h1[j] = bf16_round(gelu_f(z));
    }
    float g[CSMC_MLP_HID];
    for (int k = 0; k < CSMC_MLP_HID; ++k) {
        float z = P.b2[k];
        for (int j = 0; j < CSMC_MLP_HID; ++j) z = f_fma(h1[j], bf16_to_f(P.w2[k][j]), z);
        g[k] = gelu_f(z);
    }
    float part[CSMC_WARP];
    for (int l = 0; l < CSMC_WARP; ++l)
        part[l] = f_fma(g[l + CSMC_WARP], P.w3[l + CSMC_WARP], f_fma(g[l], P.w3[l], 0.0f));
    return clip_theta(f_add(P.b3, warp_tree_f(part)));
}

/* Multiplier of 1/rate under the proposal: e^(-theta). */
CSMC_HD float tilt_factor(float theta) { return exp2_f(f_mul(theta, -1.44269502f)); }

/* An exponential delay is tilted when its 1/rate is finite and positive. */
CSMC_HD bool tiltable(float inv) { return inv > 0.0f && inv < bits_f(0x7f800000u); }

/* 1/inv' - 1/inv: the change of one component's rate (log2 units). */
CSMC_HD double rate_change(float inv, float invp) {
    return d_sub(d_div(1.0, static_cast<double>(invp)), d_div(1.0, static_cast<double>(inv)));
}

/* Log-likelihood ratio (nominal over proposal) of one race step that took
 * time d: ln2 * d * sum_c (1/inv'_c - 1/inv_c) + [winner tilted] ln(inv'_w / inv_w)
 * (delays are -log2(u) * inv, i.e. exponential with rate ln2 / inv). */
CSMC_HD double step_log_ratio(double rate_change_sum, float d, bool win_tilted, float inv_w, float invp_w) {
    const double ln2 = 0.6931471805599453;
    double r = d_mul(d_mul(ln2, rate_change_sum), static_cast<double>(d));
    if (win_tilted)
        r = d_add(r, d_mul(ln2, log2_d(d_div(static_cast<double>(invp_w), static_cast<double>(inv_w)))));
    return r;
}

/* Training row of one location class in one step of a replayed run with CE
 * weight w: a = w * ln2 * d * sum over the class's tilted components of
 * 1/inv (nominal), b = w * [the winner is tilted and in the class].  The
 * derivative of the path's log-likelihood under the proposal with respect
 * to the class's theta is then b/w - (a/w) e^theta. */
CSMC_HD float row_a(double inv_sum, float d, float w) {
    const double ln2 = 0.6931471805599453;
    return d2f(d_mul(d_mul(d_mul(ln2, inv_sum), static_cast<double>(d)), static_cast<double>(w)));
}

/* Row record of the training set. */
struct MlpRow {
    uint16_t x[CSMC_MLP_IN];  /* BF16 features */
    float a, b;
};

}  // namespace csmc

#endif
