"""Statistical parity with the reference cuSMC binary.

tests/golden/ref_estimates.json holds estimates produced by the reference
itself (built from its sources for sm_100a, run on a B200 by
tests/golden/make_ref_estimates.py) on eight of the reference's model files
and six generated networks.  The reference cannot be compared run by run
(its random states are shared by all blocks), so the comparison is between
estimates: |ours - reference| <= eps(n_ours) + eps(n_ref) with the
Chernoff-Hoeffding half-width eps(n) = sqrt(ln(2/delta) / (2 n)),
delta = 1e-3 per comparison, for probabilities; RaceTest's deterministic
estimate must match exactly.

CPU: the oracle on a few thousand runs per case.  GPU: the CUDA kernels
(default plan) on 1e6 runs per case, a much tighter check.
"""
import json
import math
import os
import tempfile

import pytest

from conftest import GOLDEN
from cusmc_b200 import api, netgen

with open(os.path.join(GOLDEN, "ref_estimates.json")) as f:
    REF = {c["name"]: c for c in json.load(f)["cases"] if "result" in c}

DELTA = 1e-3


def eps(n):
    return math.sqrt(math.log(2 / DELTA) / (2 * n))


def case_blob(name):
    c = REF[name]
    src = c["model"]
    if src.startswith("gen:"):
        g = src[4:]
        w = {"epidemic": netgen.epidemic, "mutex_8": lambda: netgen.mutex(8), "mutex_32": lambda: netgen.mutex(32)}
        w = w.get(g, lambda: netgen.random_network(int(g.split("_")[1])))()
        with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
            f.write(w.xml)
            path = f.name
        try:
            return api.compile_model(path, c["query"][5], c["query"][2] == "-1")
        finally:
            os.unlink(path)
    with open(os.path.join(GOLDEN, "nets", f"refest_{name}.blob"), "rb") as f:
        return f.read()


def case_query(name, max_steps=0):
    T, thr, vid, mx, est, lq = REF[name]["query"]
    if vid == "-1":
        return api.location_query(float(T), max_steps=max_steps)
    return api.variable_query(int(vid), float(T), threshold=float(thr), is_max=mx == "1", is_estimate=est == "1",
                              max_steps=max_steps)


def check(name, estimate, n):
    ref = REF[name]
    if REF[name]["query"][4] == "1":  # estimate of a deterministic value
        assert estimate == pytest.approx(ref["result"], abs=1e-9)
        return
    bound = eps(n) + eps(ref["sims"])
    assert abs(estimate - ref["result"]) <= bound, (name, estimate, ref["result"], bound)


@pytest.mark.parametrize("name", sorted(REF))
def test_oracle_agrees_with_reference(name):
    import oracle
    blob = case_blob(name)
    n = 2000 if api.blob_info(blob)["n_comps"] >= 100 else 20000
    r, _, _ = oracle.run(blob, case_query(name, max_steps=1_000_000), seed=424242, n_runs=n, threads=0)
    assert r.capped == 0
    check(name, r.estimate, n)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(REF))
def test_kernel_agrees_with_reference(name):
    blob = case_blob(name)
    net = api.Network(blob)
    n = 1_000_000
    r = net.run(case_query(name, max_steps=1_000_000), seed=424242, n_runs=n)
    net.close()
    assert r.capped == 0
    check(name, r.estimate, n)
