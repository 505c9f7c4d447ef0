"""csmc_run_noalloc: the entry point for callers that cannot let the library
allocate device memory (hosts that reserve all device memory up front and
forbid later cudaMalloc/cudaFree, or whose own allocator must own every
buffer).  The caller provides the network in device memory and the output
buffers; the kernel's scratch comes from a fixed device array inside the
library.

Checked here through the C ABI: two calls in a row give, run for run, the
same flags, values and step counts as csmc_run with the thread-per-run plan
(integer and byte outputs bit-exact; the value sums equal to the last bit,
since both use the same fixed-order reduction), so the second call is not
disturbed by what the first left in the shared scratch array.  This file is
named to be collected last; it passes alone in a fresh process as well.
"""
import ctypes
import os
import tempfile

import numpy as np
import pytest

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


def _noalloc(blob, d_blob, q, seed, n, first_run=0):
    import torch
    flags = torch.zeros(n, dtype=torch.uint8, device="cuda")
    values = torch.zeros(n, dtype=torch.float64, device="cuda")
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    r = _native.Result()
    _native.check(_native.lib().csmc_run_noalloc(
        blob, d_blob.data_ptr(), len(blob), ctypes.byref(q), seed, first_run, n, flags.data_ptr(),
        values.data_ptr(), steps.data_ptr(), ctypes.byref(r), None))
    torch.cuda.synchronize()
    return r, flags.cpu().numpy(), values.cpu().numpy(), steps.cpu().numpy()


def _reference_call(blob, q, seed, n, first_run=0):
    import torch
    net = api.Network(blob)
    try:
        net.set_plan(1, 1, 1, 128)
        flags = torch.zeros(n, dtype=torch.uint8, device="cuda")
        values = torch.zeros(n, dtype=torch.float64, device="cuda")
        steps = torch.zeros(n, dtype=torch.int32, device="cuda")
        r = net.run(q, seed, n, first_run, flags=flags, values=values, steps=steps)
        return r, flags.cpu().numpy(), values.cpu().numpy(), steps.cpu().numpy()
    finally:
        net.close()


@pytest.mark.parametrize("which", ["epidemic", "random"])
def test_noalloc_matches_csmc_run_on_two_calls_in_a_row(which):
    import torch
    if which == "epidemic":
        w = netgen.epidemic()
        n = 4096
    else:
        w = netgen.random_network(3)
        n = 20000
    blob = _blob(w)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=100_000)
    # the caller owns the device copy of the network (16-byte aligned)
    d_blob = torch.frombuffer(bytearray(blob), dtype=torch.uint8).to("cuda")
    assert d_blob.data_ptr() % 16 == 0
    ref = _reference_call(blob, q, 77, n)
    for call in range(2):
        got = _noalloc(blob, d_blob, q, 77, n)
        assert np.array_equal(got[1], ref[1]), f"flags differ on call {call + 1}"
        assert np.array_equal(got[2].view(np.uint64), ref[2].view(np.uint64)), f"values differ on call {call + 1}"
        assert np.array_equal(got[3], ref[3]), f"steps differ on call {call + 1}"
        assert got[0].hits == ref[0].hits and got[0].steps == ref[0].steps and got[0].capped == ref[0].capped
        assert got[0].sum == ref[0].sum and got[0].sum_sq == ref[0].sum_sq
        assert got[0].estimate == ref[0].estimate


def test_noalloc_rejects_a_run_state_beyond_its_scratch():
    import torch
    # 2500 variables: each thread keeps 20 KB of run state, so a 128-thread
    # CTA needs 2.5 MB, beyond shared memory and beyond the 2 MiB scratch
    decl = "\n".join(f"int v{i} = 0;" for i in range(2500))
    xml = ('<?xml version="1.0" encoding="utf-8"?><nta><declaration>' + decl + '</declaration>'
           '<template><name>A</name><declaration></declaration><location id="id0"><name>L</name></location>'
           '<init ref="id0"/><transition><source ref="id0"/><target ref="id0"/>'
           '<label kind="assignment">v1 = v1 + 1</label></transition></template><system>system A;</system></nta>')
    w = netgen.Workload("many_vars", xml, var_id=1, threshold=0, horizon=10, runs=64)
    blob = _blob(w)
    d_blob = torch.frombuffer(bytearray(blob), dtype=torch.uint8).to("cuda")
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=10)
    r = _native.Result()
    n = 64
    flags = torch.zeros(n, dtype=torch.uint8, device="cuda")
    values = torch.zeros(n, dtype=torch.float64, device="cuda")
    rc = _native.lib().csmc_run_noalloc(blob, d_blob.data_ptr(), len(blob), ctypes.byref(q), 1, 0, n,
                                        flags.data_ptr(), values.data_ptr(), None, ctypes.byref(r), None)
    assert rc == _native.CSMC_ERR_LIMIT
    assert b"scratch" in _native.lib().csmc_last_error()
