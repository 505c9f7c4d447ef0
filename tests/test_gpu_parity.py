"""Bit-exact trace parity: the sm_100a kernels (verification variant, through
the C ABI) against the CPU oracle on the same seeded inputs.

For every run: the event digest (winner, delay bits, chosen edge, every
update's stored value, every broadcast receiver, in order), the final
location vector and variable bits, the step count, the goal/threshold flag
and the tracked max/min must be identical.  Clocks are compared bit for bit
too, which is stricter than the 1e-12 relative tolerance the parity target
allows.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from cusmc_b200 import api, netgen

pytestmark = pytest.mark.gpu


def _lane_shape(n_comps):
    if n_comps <= 32:
        g = 1
        while g < n_comps:
            g *= 2
        return g, 1
    k = 2
    while 32 * k < n_comps:
        k *= 2
    return 32, k


FAMILIES = [0, 1, 2, 4]


def _compare(blob, query, seed, n_runs, first_run=0, family=None):
    """family None: the library's default plan; 0: lane groups; 1: one
    thread per run; 2: one thread per run, network in global memory; 4: one
    thread per run, class-coded (skipped for networks it does not take)."""
    import oracle
    from cusmc_b200._native import CsmcError
    net = api.Network(blob)
    try:
        if family == 0:
            g, k = _lane_shape(net.info["n_comps"])
            net.set_plan(0, g, k, 256)
        elif family == 1:
            net.set_plan(1, 1, 1, 128)
        elif family == 2:
            net.set_plan(2, 1, 1, 128)
        elif family == 4:
            try:
                net.set_plan(4, 1, 1, 128)
            except CsmcError as e:
                pytest.skip(f"class-coded plan not applicable: {e}")
        r_dev, dev = net.run_verify(query, seed, n_runs, first_run)
    finally:
        net.close()
    r_cpu, cpu, _ = oracle.run(blob, query, seed, n_runs, first_run, threads=0, digests=True, final_state=True)
    for key in ("steps", "flags", "final_state", "digests"):
        a, b = dev[key], cpu[key]
        if not np.array_equal(a, b):
            bad = np.nonzero((a != b).reshape(n_runs, -1).any(axis=1))[0]
            raise AssertionError(f"{key} differs on {len(bad)} of {n_runs} runs, first run {bad[0] + first_run}")
    assert np.array_equal(dev["values"].view(np.uint64), cpu["values"].view(np.uint64))
    assert r_dev.hits == r_cpu.hits and r_dev.steps == r_cpu.steps and r_dev.capped == r_cpu.capped
    if family is not None:
        assert r_dev.family == family
    return r_dev, r_cpu


def _fixture_nets():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        man = json.load(f)
    for m in man["models"]:
        if m["generated"] or m["ref_status"] != 0:
            continue
        yield m


FIXTURE_CASES = [(m["name"], m["mode"]) for m in _fixture_nets() if m["name"] != "CSMA_100"]


@pytest.mark.parametrize("mode", ["loc", "var"])
def test_network_larger_than_shared_memory(mode):
    """CSMA_100's packed network does not fit in shared memory: the default
    plan reads it from global memory (family 2)."""
    with open(os.path.join(GOLDEN, "nets", f"CSMA_100.{mode}.blob"), "rb") as f:
        blob = f.read()
    assert len(blob) > 227 * 1024
    info = api.blob_info(blob)
    if mode == "loc":
        q = api.location_query(horizon=100, max_steps=20_000)
    else:
        q = api.variable_query(var_id=min(1, info["n_vars"] - 1), horizon=100, threshold=0, is_max=True,
                               max_steps=20_000)
    r_dev, _ = _compare(blob, q, seed=1235, n_runs=64)
    assert r_dev.family == 2


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("name,mode", FIXTURE_CASES)
def test_reference_fixtures(name, mode, family):
    with open(os.path.join(GOLDEN, "nets", f"{name}.{mode}.blob"), "rb") as f:
        blob = f.read()
    info = api.blob_info(blob)
    # a modest step cap: some fixtures never let time pass (UppaalBehaviorTest2
    # reaches an invariant bound with no enabled edge; the reference kernel
    # loops forever there) and aloha needs ~3e4 steps per run
    cap = 20_000
    if mode == "loc":
        q = api.location_query(horizon=100, max_steps=cap)
    else:
        q = api.variable_query(var_id=min(1, info["n_vars"] - 1), horizon=100, threshold=0, is_max=True,
                               max_steps=cap)
    runs = 128 if info["n_comps"] >= 100 else 512
    _compare(blob, q, seed=1235, n_runs=runs, family=family)


def _blob(w, loc=False):
    import tempfile
    with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
        f.write(w.xml)
        path = f.name
    try:
        return api.compile_model(path, w.loc_query, loc)
    finally:
        os.unlink(path)


@pytest.mark.parametrize("family", FAMILIES)
def test_epidemic_1000_runs(family):
    w = netgen.epidemic()
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    _compare(blob, q, seed=2024, n_runs=1000, family=family)


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_random_networks(seed, family):
    w = netgen.random_network(seed)
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    _compare(blob, q, seed=7 + seed, n_runs=2000, family=family)


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("n", [8, 32])
def test_mutex(n, family):
    w = netgen.mutex(n)
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    _compare(blob, q, seed=99, n_runs=500, family=family)


def test_first_run_offset_is_the_same_stream():
    w = netgen.random_network(5)
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    _compare(blob, q, seed=3, n_runs=300, first_run=1_000_000_007)


def test_step_cap_counts_capped_runs():
    w = netgen.epidemic(n_agents=20)
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=50)
    r_dev, r_cpu = _compare(blob, q, seed=11, n_runs=300)
    assert r_dev.capped > 0


def test_production_kernel_matches_verify_kernel():
    """The production variant (no digests) produces the same per-run results."""
    import torch
    w = netgen.epidemic()
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True)
    net = api.Network(blob)
    n = 4096
    flags = torch.zeros(n, dtype=torch.uint8, device="cuda")
    values = torch.zeros(n, dtype=torch.float64, device="cuda")
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    r = net.run(q, 5, n, flags=flags, values=values, steps=steps)
    r2, out = net.run_verify(q, 5, n)
    net.close()
    assert np.array_equal(flags.cpu().numpy(), out["flags"])
    assert np.array_equal(values.cpu().numpy(), out["values"])
    assert np.array_equal(steps.cpu().numpy().view(np.uint32), out["steps"])
    assert r.hits == r2.hits and r.steps == r2.steps


def _class_stress_network(kind):
    """Networks whose race classes hit the exact-race fallback often.
    ties: a class of 24 components with rate 3e38 (1/rate is a denormal
    float, so most draws give equal delays) beside a class of rate-1
    components; inf: components that move to a location whose rate program
    evaluates to 0 (1/rate = +inf), until every delay is infinite."""
    from cusmc_b200.netgen import Workload, _Doc
    d = _Doc("int hits = 0;\nint zero = 0;\nint big = 1;")
    if kind == "ties":
        for c in range(24):
            a = d.new_id()
            d.template(f"F{c}", "", [(a, "a", [("exponentialrate", "big * 3000000000000000000.0 * 100000000000000000000.0")])],
                       a, [(a, a, [("assignment", "hits = hits + 1")])])
        for c in range(8):
            a = d.new_id()
            d.template(f"S{c}", "", [(a, "a", [("exponentialrate", "1")])], a, [(a, a, [("assignment", "hits = hits + 1")])])
    else:
        for c in range(8):
            live, dead = d.new_id(), d.new_id()
            d.template(f"D{c}", "", [(live, "live", [("exponentialrate", "1")]),
                                     (dead, "dead", [("exponentialrate", "zero * 2.0")])],
                       live, [(live, dead, [("assignment", "hits = hits + 1")])])
    return Workload(f"class_{kind}", d.finish(), var_id=0, threshold=5, horizon=50, runs=256)


@pytest.mark.parametrize("family", [1, 4])
@pytest.mark.parametrize("kind", ["ties", "inf"])
def test_race_class_fallbacks(kind, family):
    import struct
    w = _class_stress_network(kind)
    blob = _blob(w)
    flags = struct.unpack_from("<I", blob, 112)[0]
    info = api.blob_info(blob)
    q = api.variable_query(0, w.horizon, threshold=w.threshold, is_max=True, max_steps=3000)
    if kind == "ties":
        # the rate program must evaluate to a finite float rate with a denormal reciprocal
        import oracle
        r, _, _ = oracle.run(blob, q, 1, 4, threads=1)
        assert r.steps > 0
    assert flags & 2, "the network should carry race classes"
    _compare(blob, q, seed=99, n_runs=256, family=family)


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("n_agents", [21, 37])
def test_epidemic_component_counts_not_a_multiple_of_four(n_agents, family):
    """The class-coded layout packs four components per word; the last
    word is partly padding here."""
    w = netgen.epidemic(n_agents=n_agents, r_threshold=n_agents // 2)
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    _compare(blob, q, seed=31, n_runs=600, family=family)


def _rate_dependency_network(kind):
    """Rate programs whose value changes without the component moving:
    clock: rates read the component's clock (the rate table must be
    evaluated every step); recv: rates read a counter that broadcast
    receivers update."""
    from cusmc_b200.netgen import Workload, _Doc
    if kind == "clock":
        d = _Doc("int hits = 0;")
        for c in range(6):
            a, b = d.new_id(), d.new_id()
            d.template(f"K{c}", "clock x;", [(a, "a", [("exponentialrate", "0.2 + x * 0.5")]),
                                             (b, "b", [("exponentialrate", "1.5")])],
                       a, [(a, b, [("guard", "x >= 1"), ("assignment", "hits = hits + 1")]),
                           (b, a, [("assignment", "x = 0")])])
    else:
        d = _Doc("int hits = 0;\nint level = 1;\nbroadcast chan go;")
        for c in range(6):
            a, b = d.new_id(), d.new_id()
            d.template(f"R{c}", "", [(a, "a", [("exponentialrate", "level * 0.3")]),
                                     (b, "b", [("exponentialrate", "2")])],
                       a, [(a, b, [("synchronisation", "go!"), ("assignment", "hits = hits + 1")]),
                           (b, a, [("synchronisation", "go?"), ("assignment", "level = level + 1")])])
    return Workload(f"rate_{kind}", d.finish(), var_id=0, threshold=5, horizon=30, runs=512)


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("kind", ["clock", "recv"])
def test_rate_programs_that_change_between_transitions(kind, family):
    import struct
    w = _rate_dependency_network(kind)
    blob = _blob(w)
    flags = struct.unpack_from("<I", blob, 112)[0]
    assert bool(flags & 4) == (kind == "recv"), "CSMC_NET_RATE_NO_CLOCK"
    q = api.variable_query(0, w.horizon, threshold=w.threshold, is_max=True, max_steps=20_000)
    _compare(blob, q, seed=5, n_runs=512, family=family)


def _philox_words(seed, run, steps, comp):
    """delay_word(seed, run, step, comp) for every step (numpy restatement of
    Philox4x32-10 on uint64 lanes)."""
    m = np.uint64(0xffffffff)
    x0 = steps.astype(np.uint64)
    x1 = np.full_like(x0, comp >> 2)
    x2 = np.full_like(x0, run & 0xffffffff)
    x3 = np.full_like(x0, run >> 32)
    k0, k1 = np.uint64(seed & 0xffffffff), np.uint64(seed >> 32)
    for r in range(10):
        p0 = np.uint64(0xD2511F53) * x0
        p1 = np.uint64(0xCD9E8D57) * x2
        x0, x1, x2, x3 = ((p1 >> np.uint64(32)) ^ x1 ^ k0) & m, p1 & m, ((p0 >> np.uint64(32)) ^ x3 ^ k1) & m, p0 & m
        k0 = (k0 + np.uint64(0x9E3779B9)) & m
        k1 = (k1 + np.uint64(0xBB67AE85)) & m
    return [x0, x1, x2, x3][comp & 3]


def test_key_zero_of_component_255():
    """In a 256-component network, component 255 has bit-reversed index 255,
    and its key is 0 when its draw is 0 (probability 2^-24 per step), the
    value that also marks an empty class.  Runs in which that happens within
    their first steps are searched for on the CPU and compared in full."""
    # (seed, run, step) triples found by the same search over seeds 1..100,
    # runs 0..29, steps 0..29999; confirmed here before use
    cases = [(66, 4, 6024), (79, 15, 3778), (100, 12, 25233)]
    w = netgen.mutex(256)
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    for seed, run, step in cases:
        word = _philox_words(seed, run, np.array([step], dtype=np.uint64), 255)[0]
        assert int(word) >> 8 == 0
        for family in (None, 1):
            _compare(blob, q, seed=seed, n_runs=1, first_run=run, family=family)
