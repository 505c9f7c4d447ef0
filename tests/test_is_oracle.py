"""Importance sampling in the CPU oracle (the checker for the GPU kernels).

* With the proposal's output layer at zero (theta = 0) a run under the
  proposal is the plain run, and its log-likelihood ratio is exactly 0.
* The estimator is unbiased: under a random (untrained) proposal the
  weighted estimate agrees with plain SMC within the two 99.9% intervals.
* The training rows of a replayed run encode its path: with CE weight 1,
  J(params) + sum(a) = -logw of the run (J = sum b*theta - a*e^theta).
* The analytic gradient agrees with finite differences of J on the FP32
  parameters.
"""
import math
import os
import tempfile

import numpy as np
import pytest

import oracle
from cusmc_b200 import api, netgen
from cusmc_b200.proposal import Proposal


def _blob(w):
    with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
        f.write(w.xml)
        path = f.name
    try:
        return api.compile_model(path)
    finally:
        os.unlink(path)


def _random_proposal(seed, out_scale=0.3):
    p = Proposal.init(seed)
    rng = np.random.default_rng(seed + 100)
    p.w3 = (rng.standard_normal(64) * out_scale / 8).astype(np.float32)
    p.b3 = 0.1
    return p


def test_zero_tilt_is_the_plain_run():
    w = netgen.epidemic(n_agents=30)
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=14, is_max=True)
    params = Proposal.init(3).pack()  # w3 = 0, b3 = 0
    out, _ = oracle.is_run(blob, q, params, 5, 200)
    _, plain, _ = oracle.run(blob, q, 5, 200, threads=0)
    assert np.array_equal(out["flags"], plain["flags"])
    assert np.array_equal(out["steps"], plain["steps"])
    assert np.array_equal(out["values"], plain["values"])
    assert np.all(out["logw"] == 0.0)


@pytest.mark.parametrize("which", ["epidemic", "epidemic_min", "random"])
def test_weighted_estimate_is_unbiased(which):
    if which == "epidemic":
        w = netgen.epidemic(n_agents=20)
        q = api.variable_query(w.var_id, 40, threshold=9, is_max=True)
    elif which == "epidemic_min":  # a min query: the susceptible count falls below 12
        w = netgen.epidemic(n_agents=20)
        q = api.variable_query(0, 40, threshold=12, is_max=False)
    else:
        w = netgen.random_network(3)
        q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    blob = _blob(w)
    n = 20000
    params = _random_proposal(7).pack()
    out, _ = oracle.is_run(blob, q, params, 11, n)
    wv = out["flags"] * np.exp(out["logw"])
    p_is, s_is = wv.mean(), wv.std() / math.sqrt(n)
    _, plain, _ = oracle.run(blob, q, 12, n, threads=0)
    p_pl = plain["flags"].mean()
    s_pl = math.sqrt(max(p_pl * (1 - p_pl), 1e-12) / n)
    assert np.any(out["logw"] != 0.0)
    assert abs(p_is - p_pl) < 3.3 * math.hypot(s_is, s_pl), (p_is, p_pl, s_is, s_pl)


def test_training_rows_encode_the_path_likelihood():
    w = netgen.epidemic(n_agents=25)
    blob = _blob(w)
    q = api.variable_query(w.var_id, 50, threshold=10, is_max=True)
    prop = _random_proposal(11)
    params = prop.pack()
    out, _ = oracle.is_run(blob, q, params, 3, 8)
    for i in range(8):
        rows = oracle.is_trace(blob, q, params, 3, [i], [1.0])
        assert len(rows) == 4 * int(out["steps"][i])
        _, J = oracle.mlp_grad(params, rows)
        lhs = J + float(rows["a"].astype(np.float64).sum())
        assert lhs == pytest.approx(-out["logw"][i], rel=2e-4, abs=2e-4)


def test_gradient_matches_finite_differences():
    w = netgen.epidemic(n_agents=25)
    blob = _blob(w)
    q = api.variable_query(w.var_id, 50, threshold=10, is_max=True)
    prop = _random_proposal(5)
    rows = oracle.is_trace(blob, q, prop.pack(), 9, list(range(6)), [0.5] * 6)
    g, J0 = oracle.mlp_grad(prop.pack(), rows)
    v = prop.vector().astype(np.float64)
    o_b1 = 64 * 16
    o_b2 = o_b1 + 64 + 64 * 64
    o_w3 = o_b2 + 64
    idx = [o_b1 + 3, o_b1 + 40, o_b2 + 7, o_b2 + 50, o_w3 + 1, o_w3 + 33, o_w3 + 64]
    for i in idx:
        h = 1e-2 * max(1.0, abs(v[i]))
        vp, vm = v.copy(), v.copy()
        vp[i] += h
        vm[i] -= h
        _, Jp = oracle.mlp_grad(Proposal.from_vector(vp).pack(), rows)
        _, Jm = oracle.mlp_grad(Proposal.from_vector(vm).pack(), rows)
        fd = (Jp - Jm) / (2 * h)
        assert g[i] == pytest.approx(fd, rel=5e-2, abs=1e-3 * max(1.0, abs(J0))), (i, g[i], fd)


def _butterfly(p):
    """csmc_mlp.h warp_tree_d: offsets 16, 8, 4, 2, 1, lane L adds lane L ^ off."""
    p = list(p)
    off = 16
    while off:
        p = [p[lane] + p[lane ^ off] for lane in range(32)]
        off //= 2
    return p[0]


def _bit_reversed_stack(p):
    """The thread-per-run importance-sampling kernel's order
    (sim_is_coded.cuh: tree_push): the lanes' partials taken in 5-bit
    bit-reversed order and merged by a five-level binary-counter stack."""
    stack = [0.0] * 5
    for i in range(32):
        v = p[int(f"{i:05b}"[::-1], 2)]
        for level in range(5):
            if not (i >> level) & 1:
                stack[level] = v
                break
            v = stack[level] + v
        else:
            return v
    raise AssertionError("unreachable")


def test_bit_reversed_stack_adds_in_the_butterfly_order():
    """FP64 sums of rate changes must carry the same bits in the one-warp and
    the one-thread-per-run kernels; float64 addition here rounds as FP64 on
    the device (round to nearest even, no fused operations)."""
    rng = np.random.default_rng(2024)
    for _ in range(5000):
        p = rng.standard_normal(32) * np.exp(rng.uniform(-40.0, 40.0, 32))
        p[rng.integers(0, 33):] = 0.0  # lanes without components add zeros
        a, b = _butterfly([float(x) for x in p]), _bit_reversed_stack([float(x) for x in p])
        assert np.float64(a).tobytes() == np.float64(b).tobytes()
