"""Batches: many (network, query) jobs in one persistent launch (csmc_batch_*).

Every job of a batch must give, run for run, exactly what csmc_run gives for
that network alone (trace digests, final states, flags, values, step counts,
hits, capped runs and value sums, bit for bit), whether the batch is launched
directly or replayed from a CUDA graph, whatever launch geometry the
autotuner picks, and with jobs that start at an offset in their run stream.
The single-network results are themselves pinned to the CPU oracle by
test_gpu_parity.py; one job here is also checked against the oracle
directly.
"""
import os
import tempfile

import numpy as np
import pytest

from cusmc_b200 import api, netgen

pytestmark = pytest.mark.gpu


def _blob(w, loc=False):
    with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
        f.write(w.xml)
        path = f.name
    try:
        return api.compile_model(path, w.loc_query, loc)
    finally:
        os.unlink(path)


def _jobs():
    """(network, query, seed, runs, first_run) for a mixed batch: sizes from
    2 to 100 components, variable and location queries, uneven run counts."""
    out = []
    specs = [
        (netgen.epidemic(), 300, 0),
        (netgen.random_network(0), 3000, 0),
        (netgen.random_network(2), 2500, 1000),
        (netgen.mutex(8), 4000, 0),
        (netgen.mutex(32), 700, 0),
        (netgen.batch_networks(count=4, base_seed=1000)[0], 1500, 0),
        (netgen.batch_networks(count=4, base_seed=1000)[3], 900, 0),
    ]
    for i, (w, runs, first) in enumerate(specs):
        blob = _blob(w)
        net = api.Network(blob)
        q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
        out.append((net, q, 7000 + i, runs, first))
    return out


def _single(net, q, seed, runs, first):
    """The same job through csmc_run_verify with the library's default plan."""
    return net.run_verify(q, seed, runs, first)


def _assert_job_equal(batch_res, batch_out, single_res, single_out):
    for key in ("flags", "steps", "digests", "final_state"):
        assert np.array_equal(np.asarray(batch_out[key]), np.asarray(single_out[key]).reshape(
            np.asarray(batch_out[key]).shape)), key
    assert np.array_equal(batch_out["values"].view(np.uint64), single_out["values"].view(np.uint64))
    assert batch_res.hits == single_res.hits
    assert batch_res.steps == single_res.steps
    assert batch_res.capped == single_res.capped
    assert batch_res.sum == single_res.sum and batch_res.sum_sq == single_res.sum_sq
    assert batch_res.estimate == single_res.estimate


@pytest.mark.parametrize("group_comps", [None, 0, 2, 64])
def test_batch_matches_single_network_runs(group_comps):
    """group_comps: the warp-per-run threshold (None: the default, 128; 0:
    every job one thread per run; 2: every job one warp per run)."""
    jobs = _jobs()
    singles = [_single(*j) for j in jobs]
    batch = api.Batch(jobs, verify=True)
    try:
        if group_comps is not None:
            batch.set_group_comps(group_comps)
        expect = sum(1 for j in jobs
                     if group_comps != 0 and (group_comps or 128) <= j[0].info["n_comps"] <= 512)
        assert batch.group_comps()[1] == expect
        for use_graph in (False, True, True):  # direct, graph capture, graph replay
            res = batch.run(use_graph=use_graph)
            for i, j in enumerate(jobs):
                _assert_job_equal(res[i], batch.outputs(i), *singles[i])
    finally:
        batch.close()
        for j in jobs:
            j[0].close()


def test_large_networks_one_warp_per_run_match_single_runs():
    """Networks of 130, 230 and 303 components (4, 8 and 16 components per
    lane in warp-per-run mode) beside small ones, against csmc_run_verify."""
    big = netgen.batch_networks(count=54, base_seed=1000)
    specs = [(big[53], 48), (big[7], 40), (big[13], 24), (netgen.mutex(8), 500), (netgen.random_network(0), 700)]
    jobs = []
    for i, (w, runs) in enumerate(specs):
        net = api.Network(_blob(w))
        q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
        jobs.append((net, q, 9100 + i, runs, 5 * i))
    singles = [_single(*j) for j in jobs]
    try:
        for k_expect, thr in ((16, 128), (16, 2)):
            batch = api.Batch(jobs, verify=True)
            try:
                batch.set_group_comps(thr)
                res = batch.run(use_graph=True)
                for i in range(len(jobs)):
                    _assert_job_equal(res[i], batch.outputs(i), *singles[i])
                    in_group = jobs[i][0].info["n_comps"] >= thr
                    assert res[i].lanes_per_run == (32 if in_group else 1)
                    if in_group:
                        assert res[i].comps_per_lane == k_expect
            finally:
                batch.close()
    finally:
        for j in jobs:
            j[0].close()


@pytest.mark.parametrize("specs,k_expect", [
    # largest network 100 components: 4 per lane
    ([("epidemic", 300), ("mutex32", 400), ("random0", 600)], 4),
    # largest 230 components: 8 per lane
    ([("big7", 40), ("mutex8", 500)], 8),
])
def test_every_lane_width_of_warp_per_run_jobs(specs, k_expect):
    """Every job one warp per run (threshold 2), with the largest network
    choosing 4 or 8 components per lane, against csmc_run_verify."""
    make = {"epidemic": netgen.epidemic, "mutex32": lambda: netgen.mutex(32), "mutex8": lambda: netgen.mutex(8),
            "random0": lambda: netgen.random_network(0),
            "big7": lambda: netgen.batch_networks(count=8, base_seed=1000)[7]}
    jobs = []
    for i, (name, runs) in enumerate(specs):
        w = make[name]()
        net = api.Network(_blob(w))
        q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
        jobs.append((net, q, 9300 + i, runs, 3 * i))
    singles = [_single(*j) for j in jobs]
    batch = api.Batch(jobs, verify=True)
    try:
        batch.set_group_comps(2)
        assert batch.group_comps() == (2, len(jobs))
        res = batch.run(use_graph=False)
        for i in range(len(jobs)):
            _assert_job_equal(res[i], batch.outputs(i), *singles[i])
            assert res[i].lanes_per_run == 32 and res[i].comps_per_lane == k_expect
    finally:
        batch.close()
        for j in jobs:
            j[0].close()


@pytest.mark.parametrize("group_comps", [0, 2])
def test_batch_job_against_the_oracle(group_comps):
    import oracle
    w = netgen.random_network(3)
    blob = _blob(w)
    net = api.Network(blob)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    other = api.Network(_blob(netgen.mutex(8)))
    q2 = api.variable_query(1, 200, threshold=1, is_max=True)
    batch = api.Batch([(other, q2, 5, 2000), (net, q, 11, 1500, 200)], verify=True)
    try:
        batch.set_group_comps(group_comps)
        res = batch.run(use_graph=True)
        out = batch.outputs(1)
        r_cpu, cpu, _ = oracle.run(blob, q, 11, 1500, 200, threads=0, digests=True, final_state=True)
        for key in ("steps", "flags", "digests"):
            assert np.array_equal(out[key], cpu[key]), key
        assert np.array_equal(out["final_state"], cpu["final_state"])
        assert np.array_equal(out["values"].view(np.uint64), cpu["values"].view(np.uint64))
        assert res[1].hits == r_cpu.hits and res[1].steps == r_cpu.steps
    finally:
        batch.close()
        net.close()
        other.close()


def test_autotuned_batch_gives_the_same_results():
    jobs = _jobs()
    batch = api.Batch(jobs, verify=False)
    try:
        before = batch.run(use_graph=False)
        threads, ctas = batch.autotune(probe_fraction=0.1)
        assert threads in (64, 128) and ctas >= 1
        assert batch.plan() == (threads, ctas)
        after = batch.run(use_graph=True)
        for a, b in zip(before, after):
            assert (a.hits, a.steps, a.capped, a.sum, a.sum_sq) == (b.hits, b.steps, b.capped, b.sum, b.sum_sq)
    finally:
        batch.close()
        for j in jobs:
            j[0].close()


def test_network_autotuner_keeps_results():
    w = netgen.epidemic()
    net = api.Network(_blob(w))
    try:
        q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True)
        ref = net.run(q, 3, 4000)
        best = net.autotune(q, 3, 4000)
        assert best.family in (0, 1, 2)
        got = net.run(q, 3, 4000)
        assert (ref.hits, ref.steps, ref.sum) == (got.hits, got.steps, got.sum)
        assert got.family == best.family
    finally:
        net.close()


def test_batch_rejects_bad_jobs():
    net = api.Network(_blob(netgen.mutex(8)))
    try:
        bad = api.variable_query(99, 10, threshold=0, is_max=True)
        with pytest.raises(api._native.CsmcError):
            api.Batch([(net, bad, 1, 10)])
    finally:
        net.close()
