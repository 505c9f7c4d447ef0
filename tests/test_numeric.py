"""The numeric primitives whose exact bits define a run, pinned against
independent references on the CPU.

The kernels and the CPU oracle compile the same definitions
(cusmc_b200/csrc/include/csmc_numeric.h, csmc_mlp.h), so bit-exact trace
parity between them says nothing about whether those definitions are right.
These tests check the definitions themselves (through the oracle's host
build of them):

* Philox4x32-10 against the published known-answer vectors of Salmon,
  Moraes, Dror and Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3"
  (SC'11; the Random123 KAT set), and against an independent Python
  restatement of the published round function on random counters and keys.
  It replaces the reference's curand XORWOW (simulation/simulation.cu:756-760).
* The float log2 of the exponential delay (the reference draws
  -__log2f(u)/rate, simulation.cu:529-530) over all 2^24 uniform draws and
  over random normal floats, against libm's log2 in double: at most 4 ulp,
  and non-decreasing in the draw (the race-class shortcut relies on it).
* The double log2 / exp2 / pow of the expression language's '^' against
  numpy (libm), with stated ulp or relative bounds.
* The proposal network's float exp2 and GELU / GELU' against float64
  evaluations of the same formulas.

Planted mistakes (restated here in numpy, never in the product): a Philox
constant with one bit flipped fails the known-answer vectors, and the float
log2 with its series one term short exceeds the 4-ulp bound.
"""
import numpy as np
import pytest

import oracle
from cusmc_b200 import _native

F32 = np.float32

# Philox4x32-10 known answers: (counter x0..x3, key k0 k1) -> output x0..x3
PHILOX_KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]

# the published constants: round multipliers and Weyl key increments
PHILOX_M0, PHILOX_M1 = 0xD2511F53, 0xCD9E8D57
PHILOX_W0, PHILOX_W1 = 0x9E3779B9, 0xBB67AE85


def philox_py(ctr, key, m0=PHILOX_M0, m1=PHILOX_M1, w0=PHILOX_W0, w1=PHILOX_W1, rounds=10):
    """Philox4x32 as published: per round, two 32x32->64 products of the
    even counter words, the odd words and the key xored into the high
    halves, then the key bumped by the Weyl constants."""
    x0, x1, x2, x3 = ctr
    k0, k1 = key
    mask = 0xffffffff
    for r in range(rounds):
        if r:
            k0, k1 = (k0 + w0) & mask, (k1 + w1) & mask
        p0, p1 = m0 * x0, m1 * x2
        x0, x1, x2, x3 = ((p1 >> 32) ^ x1 ^ k0) & mask, p1 & mask, ((p0 >> 32) ^ x3 ^ k1) & mask, p0 & mask
    return x0, x1, x2, x3


def test_philox_known_answer_vectors():
    ctr = np.array([k[0] for k in PHILOX_KAT], np.uint32)
    key = np.array([k[1] for k in PHILOX_KAT], np.uint32)
    out = oracle.numeric(_native.NUM_PHILOX, ctr, key)
    for got, (_, _, want) in zip(out, PHILOX_KAT):
        assert tuple(int(v) for v in got) == want


def test_philox_matches_published_round_function():
    rng = np.random.default_rng(7)
    n = 2000
    ctr = rng.integers(0, 2**32, size=(n, 4), dtype=np.uint64).astype(np.uint32)
    key = rng.integers(0, 2**32, size=(n, 2), dtype=np.uint64).astype(np.uint32)
    out = oracle.numeric(_native.NUM_PHILOX, ctr, key)
    for i in range(n):
        assert tuple(int(v) for v in out[i]) == philox_py(tuple(int(v) for v in ctr[i]),
                                                           tuple(int(v) for v in key[i]))


@pytest.mark.parametrize("which", ["m0", "m1", "w0", "w1", "rounds"])
def test_planted_philox_mistake_fails_the_known_answers(which):
    """The known-answer vectors pin every constant: the restatement with one
    bit of a constant flipped (or one round short) misses all three."""
    kw = {"m0": dict(m0=PHILOX_M0 ^ 0x100), "m1": dict(m1=PHILOX_M1 ^ 0x100), "w0": dict(w0=PHILOX_W0 ^ 1),
          "w1": dict(w1=PHILOX_W1 ^ 1), "rounds": dict(rounds=9)}[which]
    assert all(philox_py(c, k) == want for c, k, want in PHILOX_KAT)
    assert all(philox_py(c, k, **kw) != want for c, k, want in PHILOX_KAT)


def test_delay_stream_layout():
    """delay words: block (step, comp/4, run low, run high | 0) keyed by the
    seed, word comp % 4 (csmc_numeric.h: delay_block)."""
    seed, run, step = 0x0123456789abcdef, 0x00000002deadbeef, 77
    for comp in (0, 1, 5, 99):
        c = (step, comp >> 2, run & 0xffffffff, run >> 32)
        blk = philox_py(c, (seed & 0xffffffff, seed >> 32))
        got = oracle.numeric(_native.NUM_PHILOX, np.array([c], np.uint32),
                             np.array([(seed & 0xffffffff, seed >> 32)], np.uint32))[0]
        assert int(got[comp & 3]) == blk[comp & 3]


def _draws():
    m = np.arange(1 << 24, dtype=np.uint64)
    return ((m + 1) * np.float64(2.0 ** -24)).astype(F32)  # uniform01's exact values


def _ulp_err(got, ref):
    """|got - ref| in units of the float spacing at ref (ref nonzero)."""
    sp = np.spacing(np.abs(ref.astype(F32))).astype(np.float64)
    return np.abs(got.astype(np.float64) - ref) / sp


LOG2_ULP_BOUND = 4.0


def test_log2_of_every_uniform_draw_within_4_ulp_and_monotone():
    u = _draws()
    got = oracle.numeric(_native.NUM_LOG2_F32, u)
    ref = np.log2(u.astype(np.float64))
    assert got[-1] == 0.0 and ref[-1] == 0.0  # u = 1
    nz = ref != 0.0
    err = _ulp_err(got[nz], ref[nz])
    assert err.max() <= LOG2_ULP_BOUND, err.max()
    assert np.all(np.diff(got.astype(np.float64)) >= 0.0)


def test_log2_of_random_normal_floats_within_4_ulp():
    rng = np.random.default_rng(11)
    bits = rng.integers(0x00800000, 0x7f800000, size=2_000_000, dtype=np.uint64).astype(np.uint32)
    x = bits.view(F32)
    got = oracle.numeric(_native.NUM_LOG2_F32, x)
    ref = np.log2(x.astype(np.float64))
    nz = ref != 0.0
    assert _ulp_err(got[nz], ref[nz]).max() <= LOG2_ULP_BOUND


def _log2_restated(x, coeffs):
    """csmc_numeric.h's log2_pos restated in numpy float32 arithmetic with a
    chosen series (the fused multiply-adds through float64)."""
    b = x.view(np.uint32).astype(np.int64)
    e = ((b >> 23) & 0xff) - 127
    mb = (b & 0x7fffff) | 0x3f800000
    big = mb > 0x3fb504f3
    mb = np.where(big, mb - 0x00800000, mb)
    e = np.where(big, e + 1, e)
    m = mb.astype(np.uint32).view(F32)
    s = ((m - F32(1)) / (m + F32(1))).astype(F32)
    z = (s * s).astype(F32)
    p = np.full_like(z, F32(coeffs[0]))
    for c in coeffs[1:]:
        p = (p.astype(np.float64) * z.astype(np.float64) + np.float64(F32(c))).astype(F32)
    lm = ((s * F32(2.88539008)).astype(F32) * p).astype(F32)
    return (e.astype(F32) + lm).astype(F32)


def test_planted_short_log_series_exceeds_the_bound():
    """The restatement with the product's series reproduces the oracle bit
    for bit over all draws; with the 1/9 term dropped it breaks the bound."""
    u = _draws()
    series = [0.111111111, 0.142857143, 0.2, 0.333333333, 1.0]
    full = _log2_restated(u, series)
    assert np.array_equal(full.view(np.uint32), oracle.numeric(_native.NUM_LOG2_F32, u).view(np.uint32))
    ref = np.log2(u.astype(np.float64))
    nz = ref != 0.0
    short = _log2_restated(u, series[1:])
    assert _ulp_err(short[nz], ref[nz]).max() > LOG2_ULP_BOUND


def test_exp_delay_is_minus_log2_times_inverse_rate():
    rng = np.random.default_rng(3)
    x = rng.integers(0, 2**32, size=200_000, dtype=np.uint64).astype(np.uint32)
    inv = (1.0 / rng.uniform(0.05, 5.0, size=x.size)).astype(F32)
    got = oracle.numeric(_native.NUM_EXP_DELAY, x, inv)
    u = (((x >> 8).astype(np.float64) + 1.0) * 2.0 ** -24).astype(F32)
    l2 = oracle.numeric(_native.NUM_LOG2_F32, u)
    assert np.array_equal(got, (-l2 * inv).astype(F32))
    ref = -np.log2(u.astype(np.float64)) * inv.astype(np.float64)
    nz = ref != 0.0
    assert _ulp_err(got[nz], ref[nz]).max() <= LOG2_ULP_BOUND + 1.0


def test_log2_double_within_3_ulp():
    rng = np.random.default_rng(5)
    x = rng.integers(1, 0x7ff0000000000000, size=1_000_000, dtype=np.uint64).view(np.float64)
    x = np.concatenate([x, 1.0 + rng.uniform(-0.3, 0.3, 500_000)])
    got = oracle.numeric(_native.NUM_LOG2_F64, x)
    ref = np.log2(x)
    nz = ref != 0.0
    assert (np.abs(got - ref)[nz] / np.spacing(np.abs(ref[nz]))).max() <= 3.0
    special = np.array([0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, 5e-324, 2.2250738585072014e-308])
    with np.errstate(divide="ignore", invalid="ignore"):
        want = np.log2(special)
    np.testing.assert_array_equal(oracle.numeric(_native.NUM_LOG2_F64, special), want)


def test_exp2_double_within_1_ulp():
    rng = np.random.default_rng(6)
    t = rng.uniform(-1070.0, 1023.0, 1_000_000)
    got = oracle.numeric(_native.NUM_EXP2_F64, t)
    ref = np.exp2(t)
    ok = ref > np.finfo(np.float64).tiny
    assert (np.abs(got - ref)[ok] / np.spacing(ref[ok])).max() <= 1.0
    special = np.array([0.0, -0.0, 1024.0, -1074.0, -1080.0, -1100.0, np.nan, np.inf, -np.inf, 0.5])
    with np.errstate(over="ignore"):
        want = np.exp2(special)
    np.testing.assert_array_equal(oracle.numeric(_native.NUM_EXP2_F64, special), want)


def test_pow_bounds():
    """Non-integral exponents go through exp2(y log2 x): relative error at
    most 2^-51 (1 + |y log2 x|).  Integral exponents up to 64 use binary
    powering: at most |y| + 1 ulp."""
    rng = np.random.default_rng(8)
    eps = 2.0 ** -52
    a = np.exp(rng.uniform(-20.0, 20.0, 500_000))
    b = rng.uniform(-10.0, 10.0, 500_000)
    got = oracle.numeric(_native.NUM_POW_F64, a, b)
    ref = np.power(a, b)
    assert (np.abs(got - ref) / ref / (eps * (1.0 + np.abs(b * np.log2(a))))).max() <= 2.0
    bi = rng.integers(-64, 65, 500_000).astype(np.float64)
    ai = rng.uniform(-3.0, 3.0, 500_000)
    got = oracle.numeric(_native.NUM_POW_F64, ai, bi)
    with np.errstate(over="ignore", divide="ignore"):
        ref = np.power(ai, bi)
    fin = np.isfinite(ref) & (ref != 0.0)
    assert (np.abs(got - ref)[fin] / np.spacing(np.abs(ref[fin])) / (np.abs(bi[fin]) + 1.0)).max() <= 1.0
    assert oracle.numeric(_native.NUM_POW_F64, np.array([2.0, 0.0, -8.0]), np.array([0.0, 2.5, 1.0 / 3.0]))[
        :2].tolist() == [1.0, 0.0]


def test_proposal_exp2_and_gelu():
    rng = np.random.default_rng(9)
    t = rng.uniform(-126.0, 126.0, 1_000_000).astype(F32)
    got = oracle.numeric(_native.NUM_EXP2_F32, t).astype(np.float64)
    ref = np.exp2(t.astype(np.float64))
    assert _ulp_err(got, ref).max() <= 1.0
    x = rng.uniform(-10.0, 10.0, 1_000_000).astype(F32)
    x64 = x.astype(np.float64)
    s = 1.0 / (1.0 + np.exp(-1.5957691216057308 * (x64 + 0.044715 * x64 ** 3)))
    g = oracle.numeric(_native.NUM_GELU_F32, x).astype(np.float64)
    assert (np.abs(g - x64 * s) / (1.0 + np.abs(x64))).max() <= 4 * 2.0 ** -24
    dg = oracle.numeric(_native.NUM_GELU_GRAD_F32, x).astype(np.float64)
    dref = s + x64 * s * (1.0 - s) * 1.5957691216057308 * (1.0 + 3 * 0.044715 * x64 ** 2)
    assert (np.abs(dg - dref) / (1.0 + x64 ** 2)).max() <= 4 * 2.0 ** -24
