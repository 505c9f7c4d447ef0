"""Host logic of CE training (cusmc_b200.proposal.select_elite): the level,
the elite set, the likelihood-ratio weights, the row cap and the row offsets
that csmc_is_trace writes to, for max and min queries."""
import numpy as np
import pytest

from cusmc_b200.proposal import select_elite


def _round(n=1000, seed=0):
    rng = np.random.default_rng(seed)
    values = rng.integers(0, 100, n).astype(np.float64)
    logw = rng.normal(-3.0, 1.0, n)
    steps = rng.integers(50, 400, n).astype(np.uint32)
    return values, logw, steps


def test_level_below_the_goal_is_the_quantile():
    values, logw, steps = _round()
    e = select_elite(values, logw, steps, threshold=150.0, rho=0.1)
    q = np.quantile(values, 0.9)
    assert e.level == q and not e.at_goal
    assert set(e.runs.tolist()) == set(np.nonzero(values >= q)[0].tolist())
    # weights: normalised likelihood ratios of the elite runs
    w = np.exp(logw[e.runs] - logw[e.runs].max())
    assert np.allclose(e.weights, w / w.sum(), rtol=1e-6)
    assert e.weights.dtype == np.float32 and abs(float(e.weights.sum()) - 1.0) < 1e-5


def test_level_at_the_goal_takes_the_runs_that_reach_it():
    values, logw, steps = _round()
    e = select_elite(values, logw, steps, threshold=50.0, rho=0.1)  # half the runs exceed 50
    assert e.at_goal and e.level == pytest.approx(50.0 + 1e-9)
    assert set(e.runs.tolist()) == set(np.nonzero(values > 50.0)[0].tolist())


def test_row_offsets_are_four_rows_per_step():
    values, logw, steps = _round()
    e = select_elite(values, logw, steps, threshold=150.0)
    rows = 4 * steps[e.runs].astype(np.int64)
    assert e.n_rows == int(rows.sum())
    assert e.row_offset.dtype == np.uint64
    assert np.array_equal(e.row_offset, np.concatenate([[0], np.cumsum(rows)[:-1]]).astype(np.uint64))


def test_row_cap_keeps_the_heaviest_runs():
    values, logw, steps = _round()
    full = select_elite(values, logw, steps, threshold=150.0)
    cap = full.n_rows // 3
    e = select_elite(values, logw, steps, threshold=150.0, max_rows=cap)
    assert 0 < e.n_rows <= cap and len(e.runs) < len(full.runs)
    kept = set(e.runs.tolist())
    dropped = [r for r in full.runs.tolist() if r not in kept]
    assert min(logw[list(kept)]) >= max(logw[dropped]) - 1e-12
    # a cap below every run still keeps one run
    one = select_elite(values, logw, steps, threshold=150.0, max_rows=1)
    assert len(one.runs) == 1 and abs(float(one.weights[0]) - 1.0) < 1e-6


def test_min_query_mirrors_the_max_query():
    values, logw, steps = _round()
    hi = select_elite(values, logw, steps, threshold=60.0, is_max=True, rho=0.2)
    lo = select_elite(-values, logw, steps, threshold=-60.0, is_max=False, rho=0.2)
    assert np.array_equal(np.sort(hi.runs), np.sort(lo.runs))
    assert lo.level == pytest.approx(-hi.level) and lo.at_goal == hi.at_goal


def test_weights_stay_finite_for_tiny_likelihood_ratios():
    values, logw, steps = _round()
    e = select_elite(values, logw - 5000.0, steps, threshold=150.0)
    assert np.all(np.isfinite(e.weights)) and abs(float(e.weights.sum()) - 1.0) < 1e-5


def test_library_init_and_pack():
    """csmc_mlp_init starts at theta = 0 (zero output layer, zero biases);
    csmc_mlp_pack packs a master vector as Proposal.pack does (host code of
    the library, no GPU)."""
    import ctypes
    import math
    from cusmc_b200 import _native
    from cusmc_b200 import proposal as P
    p = P.init_c(7)
    assert not p.w3.any() and p.b3 == 0.0 and not p.b1.any() and not p.b2.any() and not p.w1[:, 10:].any()
    assert 0.5 < float(np.std(p.w1[:, :10])) / math.sqrt(0.2) < 1.5
    assert 0.8 < float(np.std(p.w2)) / math.sqrt(2.0 / 64) < 1.2
    assert np.array_equal(P.init_c(7).vector(), p.vector()) and not np.array_equal(P.init_c(8).vector(), p.vector())
    r = P.Proposal.init(3)
    rng = np.random.default_rng(5)
    r.w3 = rng.standard_normal(64).astype(np.float32)
    r.b3 = 0.25
    r.b1 = rng.standard_normal(64).astype(np.float32)
    buf = ctypes.create_string_buffer(P.PARAM_BYTES)
    x = r.vector()
    _native.check(_native.lib().csmc_mlp_pack(x.ctypes.data, buf))
    assert buf.raw == r.pack()


def test_selection_fallback_and_min_query():
    """No run reaches the level (all scores equal to the quantile is not
    possible here): the highest-scoring runs are taken; a min query negates
    the scores and reports the level in value units."""
    values = np.array([5.0, 1.0, 3.0, 2.0, 4.0] * 40)
    logw = np.zeros(values.size)
    steps = np.full(values.size, 10, np.uint32)
    e = select_elite(values, logw, steps, threshold=2.5, is_max=False, rho=0.1)
    assert e.at_goal and np.all(values[e.runs] < 2.5)
    assert e.level == pytest.approx(2.5 - 1e-9)
    assert abs(float(e.weights.sum()) - 1.0) < 1e-6
