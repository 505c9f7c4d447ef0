"""The benchmark's full-size workload (1e6 epidemic runs per launch) checked
through properties that do not depend on the launch size:

* run-index keying: runs sampled from the 1e6-run launch equal the same
  runs simulated alone (the class-coded kernel on small launches) and the
  CPU oracle's, bit for bit;
* a sum of sums: the launch's hits, steps and per-run flags and values are
  the sums of ten launches of 1e5 runs over the same run range, and its
  estimate is its mean of flags;
* the estimate agrees with the reference binary's estimate for the same
  query within the Chernoff-Hoeffding bound of the two run counts
  (tests/golden/ref_estimates.json).
"""
import json
import math
import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN
from cusmc_b200 import api, netgen

pytestmark = pytest.mark.gpu

N = 1_000_000
SEED = 1235


def _epidemic():
    w = netgen.epidemic()
    with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
        f.write(w.xml)
        path = f.name
    try:
        blob = api.compile_model(path)
    finally:
        os.unlink(path)
    return w, blob, api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True)


def test_full_size_launch_keeps_runs_and_sums():
    import torch
    import oracle
    w, blob, q = _epidemic()
    dev = torch.device("cuda")
    net = api.Network(blob)
    try:
        flags = torch.empty(N, dtype=torch.uint8, device=dev)
        values = torch.empty(N, dtype=torch.float64, device=dev)
        steps = torch.empty(N, dtype=torch.int32, device=dev)
        r = net.run(q, SEED, N, 0, flags=flags, values=values, steps=steps)
        f_all, v_all, s_all = flags.cpu().numpy(), values.cpu().numpy(), steps.cpu().numpy().view(np.uint32)
        assert r.runs == N and r.hits == int(f_all.sum()) and r.steps == int(s_all.sum(dtype=np.uint64))
        assert r.estimate == r.hits / N
        # ten launches of 1e5 runs over the same range: the same runs
        hits = steps_total = 0
        chunk = N // 10
        for k in range(10):
            fc = torch.empty(chunk, dtype=torch.uint8, device=dev)
            vc = torch.empty(chunk, dtype=torch.float64, device=dev)
            sc = torch.empty(chunk, dtype=torch.int32, device=dev)
            rc = net.run(q, SEED, chunk, k * chunk, flags=fc, values=vc, steps=sc)
            hits += rc.hits
            steps_total += rc.steps
            assert np.array_equal(fc.cpu().numpy(), f_all[k * chunk:(k + 1) * chunk])
            assert np.array_equal(vc.cpu().numpy().view(np.uint64), v_all[k * chunk:(k + 1) * chunk].view(np.uint64))
            assert np.array_equal(sc.cpu().numpy().view(np.uint32), s_all[k * chunk:(k + 1) * chunk])
        assert hits == r.hits and steps_total == r.steps
    finally:
        net.close()
    # sampled runs of the full launch against the oracle
    for first in (0, 333_333, 999_488):
        _, cpu, _ = oracle.run(blob, q, SEED, 512, first, threads=0)
        assert np.array_equal(cpu["flags"], f_all[first:first + 512])
        assert np.array_equal(cpu["steps"], s_all[first:first + 512])
        assert np.array_equal(cpu["values"].view(np.uint64), v_all[first:first + 512].view(np.uint64))


def test_full_size_estimate_agrees_with_the_reference():
    with open(os.path.join(GOLDEN, "ref_estimates.json")) as f:
        cases = json.load(f)["cases"]
    c = next(c for c in cases if c["name"] == "epidemic_100")
    w, blob, q = _epidemic()
    # the same query: Pr[<=T](<> R > threshold) on variable 3
    assert c["query"][:4] == [str(w.horizon), str(w.threshold), str(w.var_id), "1"]
    net = api.Network(blob)
    try:
        r = net.run(q, SEED, N, 0)
    finally:
        net.close()
    eps = math.sqrt(math.log(2 / 1e-3) / (2 * N)) + math.sqrt(math.log(2 / 1e-3) / (2 * c["sims"]))
    assert abs(r.estimate - c["result"]) <= eps
