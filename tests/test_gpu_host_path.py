"""csmc_run_host, the host-buffer entry point: per-run outputs and sums equal
to csmc_run on device buffers and to the CPU oracle, across repeated calls
with the same network (the cached plan and buffers), alternating networks,
a copy-back spanning several staging chunks, and after releasing the
cached state (csmc_run_host_release)."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

import oracle
from cusmc_b200 import _native, api, netgen

pytestmark = pytest.mark.gpu


def _blob(w):
    with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
        f.write(w.xml)
        path = f.name
    try:
        return api.compile_model(path)
    finally:
        os.unlink(path)


def _device_run(blob, q, seed, n, first_run=0):
    import torch
    net = api.Network(blob)
    try:
        flags = torch.zeros(n, dtype=torch.uint8, device="cuda")
        values = torch.zeros(n, dtype=torch.float64, device="cuda")
        steps = torch.zeros(n, dtype=torch.int32, device="cuda")
        r = net.run(q, seed, n, first_run, flags=flags, values=values, steps=steps)
        return r, flags.cpu().numpy(), values.cpu().numpy(), steps.cpu().numpy().view(np.uint32)
    finally:
        net.close()


def _check(got, want):
    r, flags, values, steps = got
    rw, fw, vw, sw = want
    assert np.array_equal(flags, fw)
    assert np.array_equal(values.view(np.uint64), vw.view(np.uint64))
    if steps is not None:
        assert np.array_equal(steps, sw)
    assert (r.hits, r.steps, r.capped) == (rw.hits, rw.steps, rw.capped)
    # host sums in run order
    s = s2 = 0.0
    for v in vw.tolist():
        s += v
        s2 += v * v
    assert r.sum == s and r.sum_sq == s2


def test_run_host_repeated_and_alternating_networks():
    epi, rnd = netgen.epidemic(), netgen.random_network(4)
    b_epi, b_rnd = _blob(epi), _blob(rnd)
    q_epi = api.variable_query(epi.var_id, epi.horizon, threshold=epi.threshold, is_max=True)
    q_rnd = api.variable_query(rnd.var_id, rnd.horizon, threshold=rnd.threshold, is_max=True, max_steps=100_000)
    want_epi = _device_run(b_epi, q_epi, 5, 3000, 17)
    want_rnd = _device_run(b_rnd, q_rnd, 6, 5000)
    for _ in range(2):
        _check(api.run_host(b_epi, q_epi, 5, 3000, 17, want_steps=True), want_epi)
    _check(api.run_host(b_rnd, q_rnd, 6, 5000, want_steps=True), want_rnd)
    _check(api.run_host(b_epi, q_epi, 5, 3000, 17), want_epi[:3] + (None,))
    # the oracle on a prefix
    r_cpu, cpu, _ = oracle.run(b_epi, q_epi, 5, 256, first_run=17, threads=0)
    r, flags, values, _ = api.run_host(b_epi, q_epi, 5, 256, 17)
    assert np.array_equal(flags, cpu["flags"]) and np.array_equal(values.view(np.uint64),
                                                                 cpu["values"].view(np.uint64))


def test_run_host_copy_back_over_several_chunks_into_caller_buffers():
    w = netgen.random_network(9)
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    n = 1_300_000  # 10.4 MB of values: three 4 MB staging chunks
    want = _device_run(blob, q, 3, n)
    flags = np.full(n + 7, 0xAB, np.uint8)
    values = np.full(n + 7, -1.0)
    steps = np.zeros(n + 7, np.uint32)
    got = api.run_host(blob, q, 3, n, out=(flags, values, steps))
    _check((got[0], flags[:n], values[:n], steps[:n]), want)
    assert np.all(flags[n:] == 0xAB) and np.all(values[n:] == -1.0)  # nothing written past n


def test_run_host_after_release_and_with_no_outputs():
    w = netgen.epidemic()
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True)
    want = _device_run(blob, q, 8, 2000)
    _check(api.run_host(blob, q, 8, 2000), want[:3] + (None,))
    _native.lib().csmc_run_host_release()
    _check(api.run_host(blob, q, 8, 2000), want[:3] + (None,))
    # no host outputs at all: the sums still come from every run's value
    r = api.Result()
    _native.check(_native.lib().csmc_run_host(blob, len(blob), ctypes.byref(q), 8, 0, 2000, None, None, None,
                                              ctypes.byref(r)))
    s = 0.0
    for v in want[2].tolist():
        s += v
    assert r.hits == want[0].hits and r.sum == s
    assert api.run_host(blob, q, 8, 0)[0].runs == 0
