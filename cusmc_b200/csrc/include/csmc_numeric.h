/*
 * Numeric building blocks whose exact bits define a run: the counter-based
 * random stream, the uniform maps, the logarithm used for exponential delays
 * and the power function.  Compiled unchanged for the host (CPU oracle, CLI)
 * and the device (kernels) so that both produce identical bits.  Every
 * operation is an IEEE-754 basic operation with round-to-nearest (add, sub,
 * mul, div, sqrt, fused multiply-add) written out explicitly: on the device
 * through the __*_rn intrinsics, which the compiler never contracts or
 * reorders; on the host through plain operators compiled with
 * -ffp-contract=off and std::fma.
 *
 * Random stream: Philox4x32-10 (J. Salmon, M. Moraes, R. Dror, D. Shaw,
 * "Parallel Random Numbers: As Easy as 1, 2, 3", SC'11), multipliers
 * 0xD2511F53/0xCD9E8D57 and Weyl key increments 0x9E3779B9/0xBB67AE85 as
 * published there.  Key = 64-bit seed; counter = (step, slot, run low, run
 * high | stream bit).  It replaces the reference's curand XORWOW states
 * (simulation/simulation.cu:756-760), which are shared by all blocks and make
 * the reference's runs irreproducible.
 *
 * Logarithm: ln(m) = 2 atanh(s), s = (m-1)/(m+1), m in [sqrt(1/2), sqrt(2))
 * (Abramowitz & Stegun 4.1.27), evaluated with a fixed number of series terms.
 */
#ifndef CSMC_NUMERIC_H
#define CSMC_NUMERIC_H

#include <stdint.h>

#include <cmath>
#include <cstring>

#if defined(__CUDACC__)
#define CSMC_HD __host__ __device__ __forceinline__
#else
#define CSMC_HD inline
#endif

namespace csmc {

// ---- exact basic operations ------------------------------------------------
CSMC_HD float f_add(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
CSMC_HD float f_mul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
CSMC_HD float f_div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
CSMC_HD float f_fma(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
CSMC_HD double d_add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
CSMC_HD double d_sub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
CSMC_HD double d_mul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
CSMC_HD double d_div(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
CSMC_HD double d_fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
CSMC_HD double d_sqrt(double a) {
#ifdef __CUDA_ARCH__
    return __dsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}
CSMC_HD float d2f(double a) {  // round to nearest
#ifdef __CUDA_ARCH__
    return __double2float_rn(a);
#else
    return static_cast<float>(a);
#endif
}
CSMC_HD uint32_t f_bits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
#endif
}
CSMC_HD float bits_f(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}
CSMC_HD uint64_t d_bits(double d) {
#ifdef __CUDA_ARCH__
    return static_cast<uint64_t>(__double_as_longlong(d));
#else
    uint64_t u;
    std::memcpy(&u, &d, 8);
    return u;
#endif
}
CSMC_HD double bits_d(uint64_t u) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double(static_cast<long long>(u));
#else
    double d;
    std::memcpy(&d, &u, 8);
    return d;
#endif
}
CSMC_HD bool d_isnan(double x) { return x != x; }

// Truncating double -> int that saturates and maps NaN to 0 (the device
// conversion instruction's behaviour, written out for the host).
CSMC_HD int d2i_sat(double x) {
#ifdef __CUDA_ARCH__
    return __double2int_rz(x);
#else
    if (x != x) return 0;
    if (x >= 2147483647.0) return 2147483647;
    if (x <= -2147483648.0) return -2147483647 - 1;
    return static_cast<int>(x);
#endif
}
CSMC_HD int f2i_sat(float x) {
#ifdef __CUDA_ARCH__
    return __float2int_rz(x);
#else
    if (x != x) return 0;
    if (x >= 2147483647.0f) return 2147483647;
    if (x <= -2147483648.0f) return -2147483647 - 1;
    return static_cast<int>(x);
#endif
}

// ---- Philox4x32-10 -----------------------------------------------------------
struct u32x4 {
    uint32_t x, y, z, w;
};

// 32 x 32 -> 64-bit product split into halves (one wide multiply).
CSMC_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
    const uint64_t p = static_cast<uint64_t>(a) * static_cast<uint64_t>(b);
    lo = static_cast<uint32_t>(p);
    hi = static_cast<uint32_t>(p >> 32);
}

CSMC_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c.x, hi0, lo0);
        mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
        u32x4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Stream layout.  Delay draws: one 32-bit word per (run, step, component);
// four consecutive components share one Philox block.  Choice draws (edge
// selection when several edges are enabled): word 0 for the race winner,
// word 1 for a broadcast receiver, block (step, component) of stream 1.
#define CSMC_STREAM_CHOICE 0x80000000u

CSMC_HD u32x4 delay_block(uint64_t seed, uint64_t run, uint32_t step, uint32_t comp_group) {
    u32x4 c{step, comp_group, static_cast<uint32_t>(run), static_cast<uint32_t>(run >> 32)};
    return philox4x32_10(c, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
}

// The delay blocks of one race step share every counter word but the
// component group q: counter (step, q, run low, run high), key = seed.  The
// parts of rounds 1-3 that depend only on the shared words are computed once
// per step (philox_step); philox_block(q) finishes the block.  The integer
// operations are those of philox4x32_10 regrouped, so the bits are equal.
// Round keys: k0 + r * 0x9E3779B9, k1 + r * 0xBB67AE85 for rounds r = 0..9.
struct PhiloxKeys {
    uint32_t k0[10], k1[10];
};

CSMC_HD PhiloxKeys philox_keys(uint64_t seed) {
    PhiloxKeys K;
    uint32_t a = static_cast<uint32_t>(seed), b = static_cast<uint32_t>(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        K.k0[r] = a;
        K.k1[r] = b;
        a += 0x9E3779B9u;
        b += 0xBB67AE85u;
    }
    return K;
}

struct PhiloxStep {
    uint32_t a1;  // round 1: x = a1 ^ q
    uint32_t c2;  // round 2: z = hi(M0 * x1) ^ c2
    uint32_t d3;  // round 3: x = hi(M1 * z2) ^ d3
    uint32_t b3;  // round 3: z = b3 ^ lo(M0 * x1)
    uint32_t w3;  // round 3: w
};

CSMC_HD PhiloxStep philox_step(const PhiloxKeys &K, uint32_t step, uint64_t run) {
    uint32_t h0, l0, h1, l1;
    mulhilo32(0xD2511F53u, step, h0, l0);
    mulhilo32(0xCD9E8D57u, static_cast<uint32_t>(run), h1, l1);
    // after round 1: x1 = h1 ^ q ^ k0[0], y1 = l1, z1 = h0 ^ run_hi ^ k1[0], w1 = l0
    const uint32_t y1 = l1, z1 = h0 ^ static_cast<uint32_t>(run >> 32) ^ K.k1[0], w1 = l0;
    PhiloxStep s;
    s.a1 = h1 ^ K.k0[0];
    // round 2: the z1 product is shared; x2 and y2 are shared
    uint32_t g1, g0;
    mulhilo32(0xCD9E8D57u, z1, g1, g0);
    const uint32_t x2 = g1 ^ y1 ^ K.k0[1], y2 = g0;
    s.c2 = w1 ^ K.k1[1];
    // round 3: the x2 product is shared
    uint32_t p1, p0;
    mulhilo32(0xD2511F53u, x2, p1, p0);
    s.d3 = y2 ^ K.k0[2];
    s.b3 = p1 ^ K.k1[2];
    s.w3 = p0;
    return s;
}

CSMC_HD u32x4 philox_block(const PhiloxKeys &K, const PhiloxStep &s, uint32_t q) {
    uint32_t h0, l0, h1, l1;
    mulhilo32(0xD2511F53u, s.a1 ^ q, h0, l0);         // round 2, the x1 product
    const uint32_t z2 = h0 ^ s.c2, w2 = l0;
    mulhilo32(0xCD9E8D57u, z2, h1, l1);               // round 3, the z2 product
    u32x4 c{h1 ^ s.d3, l1, s.b3 ^ w2, s.w3};
#pragma unroll
    for (int r = 3; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c.x, hi0, lo0);
        mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
        c = u32x4{hi1 ^ c.y ^ K.k0[r], lo1, hi0 ^ c.w ^ K.k1[r], lo0};
    }
    return c;
}

CSMC_HD uint32_t word_of(const u32x4 &b, uint32_t i) {
    return i == 0 ? b.x : i == 1 ? b.y : i == 2 ? b.z : b.w;
}

CSMC_HD uint32_t delay_word(uint64_t seed, uint64_t run, uint32_t step, uint32_t comp) {
    return word_of(delay_block(seed, run, step, comp >> 2), comp & 3u);
}

CSMC_HD uint32_t choice_word(uint64_t seed, uint64_t run, uint32_t step, uint32_t comp, uint32_t which) {
    u32x4 c{step, comp, static_cast<uint32_t>(run), static_cast<uint32_t>(run >> 32) | CSMC_STREAM_CHOICE};
    return word_of(philox4x32_10(c, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32)), which);
}

// Uniform float in (0, 1]: ((x >> 8) + 1) * 2^-24, exact.
CSMC_HD float uniform01(uint32_t x) { return f_mul(static_cast<float>((x >> 8) + 1u), 5.9604644775390625e-08f); }

// ---- log2 of a positive normal float ------------------------------------------
CSMC_HD float log2_pos(float x) {
    uint32_t b = f_bits(x);
    int e = static_cast<int>((b >> 23) & 0xffu) - 127;
    uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;  // m in [1, 2)
    if (mb > 0x3fb504f3u) {                         // m > sqrt(2): halve m exactly
        mb -= 0x00800000u;
        e += 1;
    }
    const float m = bits_f(mb);
    const float s = f_div(f_add(m, -1.0f), f_add(m, 1.0f));
    const float z = f_mul(s, s);
    float p = 0.111111111f;        // 1/9
    p = f_fma(p, z, 0.142857143f);  // 1/7
    p = f_fma(p, z, 0.2f);          // 1/5
    p = f_fma(p, z, 0.333333333f);  // 1/3
    p = f_fma(p, z, 1.0f);
    // log2(m) = (2 / ln 2) * s * p
    const float lm = f_mul(f_mul(s, 2.88539008f), p);
    return f_add(static_cast<float>(e), lm);
}

// Reciprocal of an exponential rate as the delay formula uses it: the rate
// rounded to float, then 1/rate correctly rounded.
CSMC_HD float inv_rate(double rate) { return f_div(1.0f, d2f(rate)); }

// Exponential delay: -log2(u) / rate, as the reference draws it
// (simulation/simulation.cu:529-530: effective rate is rate * ln 2), computed
// as -log2(u) * (1/rate) with the reciprocal above.
CSMC_HD float exp_delay(uint32_t x, float inv) {
    const float u = uniform01(x);
    const float l = log2_pos(u);
    return f_mul(-l, inv);
}

// Uniform delay on (0, max]: max * u in double, stored as float
// (simulation/simulation.cu:514-516).
CSMC_HD float uniform_delay(uint32_t x, double max_delay) {
    return d2f(d_mul(max_delay, static_cast<double>(uniform01(x))));
}

// ---- double log2 / exp2 / pow (for the '^' operator) ----------------------------
CSMC_HD double log2_d(double x) {
    if (d_isnan(x) || x < 0.0) return bits_d(0x7ff8000000000000ull);
    if (x == 0.0) return -bits_d(0x7ff0000000000000ull);
    if (x == bits_d(0x7ff0000000000000ull)) return x;
    uint64_t b = d_bits(x);
    int e = static_cast<int>((b >> 52) & 0x7ffu);
    if (e == 0) {  // subnormal: scale up by 2^64
        x = d_mul(x, 18446744073709551616.0);
        b = d_bits(x);
        e = static_cast<int>((b >> 52) & 0x7ffu) - 64;
    }
    e -= 1023;
    uint64_t mb = (b & 0xfffffffffffffull) | 0x3ff0000000000000ull;
    if (mb > 0x3ff6a09e667f3bcdull) {
        mb -= 0x0010000000000000ull;
        e += 1;
    }
    const double m = bits_d(mb);
    const double s = d_div(d_sub(m, 1.0), d_add(m, 1.0));
    const double z = d_mul(s, s);
    double p = 1.0 / 23.0;
    p = d_fma(p, z, 1.0 / 21.0);
    p = d_fma(p, z, 1.0 / 19.0);
    p = d_fma(p, z, 1.0 / 17.0);
    p = d_fma(p, z, 1.0 / 15.0);
    p = d_fma(p, z, 1.0 / 13.0);
    p = d_fma(p, z, 1.0 / 11.0);
    p = d_fma(p, z, 1.0 / 9.0);
    p = d_fma(p, z, 1.0 / 7.0);
    p = d_fma(p, z, 1.0 / 5.0);
    p = d_fma(p, z, 1.0 / 3.0);
    p = d_fma(p, z, 1.0);
    const double lm = d_mul(d_mul(s, 2.8853900817779268), p);  // 2/ln 2
    return d_add(static_cast<double>(e), lm);
}

CSMC_HD double exp2_d(double t) {
    if (d_isnan(t)) return t;
    if (t > 1024.0) return bits_d(0x7ff0000000000000ull);
    if (t < -1080.0) return 0.0;
    // n = nearest integer, f in [-0.5, 0.5]
    double n = t >= 0.0 ? static_cast<double>(static_cast<long long>(d_add(t, 0.5)))
                        : -static_cast<double>(static_cast<long long>(d_add(-t, 0.5)));
    const double f = d_sub(t, n);
    const double w = d_mul(f, 0.69314718055994531);  // ln 2
    // e^w by Taylor series, 17 terms, Horner form
    double p = 1.0 / 355687428096000.0;  // 1/17!
    const double inv[] = {1.0 / 20922789888000.0, 1.0 / 1307674368000.0, 1.0 / 87178291200.0,
                          1.0 / 6227020800.0,     1.0 / 479001600.0,     1.0 / 39916800.0,
                          1.0 / 3628800.0,        1.0 / 362880.0,        1.0 / 40320.0,
                          1.0 / 5040.0,           1.0 / 720.0,           1.0 / 120.0,
                          1.0 / 24.0,             1.0 / 6.0,             0.5,
                          1.0,                    1.0};
    for (int i = 0; i < 17; ++i) p = d_fma(p, w, inv[i]);
    int ni = static_cast<int>(n);
    // scale by 2^ni in at most two exact steps
    double r = p;
    while (ni > 1000) { r = d_mul(r, bits_d(static_cast<uint64_t>(1023 + 1000) << 52)); ni -= 1000; }
    while (ni < -1000) { r = d_mul(r, bits_d(static_cast<uint64_t>(1023 - 1000) << 52)); ni += 1000; }
    return d_mul(r, bits_d(static_cast<uint64_t>(1023 + ni) << 52));
}

// x^y for the model language's '^': integral exponents by binary powering,
// others through exp2(y * log2(x)).
CSMC_HD double pow_model(double x, double y) {
    if (y == 0.0) return 1.0;
    if (x == 1.0) return 1.0;
    if (d_isnan(x) || d_isnan(y)) return bits_d(0x7ff8000000000000ull);
    const double ay = y < 0.0 ? -y : y;
    if (ay <= 64.0 && static_cast<double>(static_cast<int>(ay)) == ay) {
        int k = static_cast<int>(ay);
        double r = 1.0, b = x;
        while (k) {
            if (k & 1) r = d_mul(r, b);
            b = d_mul(b, b);
            k >>= 1;
        }
        return y < 0.0 ? d_div(1.0, r) : r;
    }
    if (x == 0.0) return y > 0.0 ? 0.0 : bits_d(0x7ff0000000000000ull);
    if (x < 0.0) {
        // only integral exponents are defined for negative bases
        const double fy = static_cast<double>(static_cast<long long>(y));
        if (fy != y) return bits_d(0x7ff8000000000000ull);
        const double r = exp2_d(d_mul(y, log2_d(-x)));
        const long long iy = static_cast<long long>(y);
        return (iy & 1) ? -r : r;
    }
    return exp2_d(d_mul(y, log2_d(x)));
}

// ---- race keys --------------------------------------------------------------------
// Order-preserving 32-bit key of a float delay; -0 equals +0 and NaN sorts
// after +inf (a NaN delay never wins).
CSMC_HD uint32_t delay_key(float d) {
    if (d != d) return 0xffffffffu;
    if (d == 0.0f) return 0x80000000u;
    const uint32_t b = f_bits(d);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// The reference's shared-memory tree argmin (simulation/simulation.cu:
// 576-628, stride halving, strict '<') returns, among equal minima, the
// component whose index has the smallest bit-reversal over log2 of the
// padded width.  The kernels reduce on (key, bitrev(index)).
CSMC_HD uint32_t bitrev_bits(uint32_t i, uint32_t bits) {
    if (bits == 0) return 0;
#ifdef __CUDA_ARCH__
    return __brev(i) >> (32u - bits);
#else
    uint32_t r = 0;
    for (uint32_t k = 0; k < bits; ++k) r |= ((i >> k) & 1u) << (bits - 1 - k);
    return r;
#endif
}

CSMC_HD uint32_t ceil_log2(uint32_t n) {
    uint32_t b = 0;
    while ((1u << b) < n) ++b;
    return b;
}

}  // namespace csmc

#endif
