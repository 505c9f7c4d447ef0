"""The device copies of the numeric primitives against the host copies, bit
for bit (csmc_numeric_eval through the C ABI against the CPU oracle's build
of the same definitions): Philox4x32-10 on random counters and keys and on
the published known-answer vectors, the float log2 on every one of the 2^24
uniform draws, the exponential delay, the double log2/exp2/pow with special
values, and the proposal network's exp2 and GELU.  The CPU tests of
test_numeric.py pin the host copies against independent references."""
import ctypes

import numpy as np
import pytest

import oracle
from cusmc_b200 import _native

pytestmark = pytest.mark.gpu


def _device_eval(fn, a, b=None):
    import torch
    a = np.ascontiguousarray(a)
    n = a.shape[0]
    da = torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()
    db = None if b is None else torch.from_numpy(np.ascontiguousarray(b).view(np.uint8).reshape(-1).copy()).cuda()
    want = oracle.numeric(fn, a, b)
    out = torch.zeros(want.nbytes, dtype=torch.uint8, device="cuda")
    _native.check(_native.lib().csmc_numeric_eval(fn, ctypes.c_void_p(da.data_ptr()),
                                                  None if db is None else ctypes.c_void_p(db.data_ptr()), n,
                                                  ctypes.c_void_p(out.data_ptr()), None))
    got = out.cpu().numpy().view(want.dtype).reshape(want.shape)
    return got, want


def _same_bits(got, want):
    w = {4: np.uint32, 8: np.uint64}[want.dtype.itemsize]
    return np.array_equal(got.view(w), want.view(w))


def test_device_philox_equals_host():
    from test_numeric import PHILOX_KAT
    rng = np.random.default_rng(21)
    ctr = rng.integers(0, 2**32, size=(1 << 20, 4), dtype=np.uint64).astype(np.uint32)
    key = rng.integers(0, 2**32, size=(1 << 20, 2), dtype=np.uint64).astype(np.uint32)
    ctr[:3] = [k[0] for k in PHILOX_KAT]
    key[:3] = [k[1] for k in PHILOX_KAT]
    got, want = _device_eval(_native.NUM_PHILOX, ctr, key)
    assert np.array_equal(got, want)
    for i, (_, _, kat) in enumerate(PHILOX_KAT):
        assert tuple(int(v) for v in got[i]) == kat


def test_device_log2_of_every_draw_equals_host():
    m = np.arange(1 << 24, dtype=np.uint64)
    u = ((m + 1) * np.float64(2.0 ** -24)).astype(np.float32)
    got, want = _device_eval(_native.NUM_LOG2_F32, u)
    assert _same_bits(got, want)


def test_device_exp_delay_equals_host():
    rng = np.random.default_rng(22)
    x = rng.integers(0, 2**32, size=1 << 20, dtype=np.uint64).astype(np.uint32)
    inv = (1.0 / rng.uniform(0.01, 10.0, size=x.size)).astype(np.float32)
    inv[:4] = [np.inf, 0.0, np.float32(1e-30), np.float32(3e38)]
    got, want = _device_eval(_native.NUM_EXP_DELAY, x, inv)
    assert _same_bits(got, want)


def _doubles(rng, n):
    x = rng.integers(0, 2**64, size=n, dtype=np.uint64).view(np.float64)
    special = np.array([0.0, -0.0, 1.0, -1.0, 0.5, 2.0, np.inf, -np.inf, np.nan, 5e-324, 2.2250738585072014e-308,
                        1.7976931348623157e308, 1024.0, -1074.0, -1080.0])
    x[:special.size] = special
    return x


def test_device_double_functions_equal_host():
    rng = np.random.default_rng(23)
    x = _doubles(rng, 1 << 19)
    for fn in (_native.NUM_LOG2_F64, _native.NUM_EXP2_F64):
        got, want = _device_eval(fn, x)
        assert _same_bits(got, want), fn
    t = rng.uniform(-1100.0, 1100.0, 1 << 19)
    got, want = _device_eval(_native.NUM_EXP2_F64, t)
    assert _same_bits(got, want)
    a = np.concatenate([_doubles(rng, 1 << 18), rng.uniform(-5.0, 5.0, 1 << 18)])
    b = np.concatenate([_doubles(rng, 1 << 18), rng.integers(-70, 71, 1 << 18).astype(np.float64)])
    got, want = _device_eval(_native.NUM_POW_F64, a, b)
    assert _same_bits(got, want)


def test_device_proposal_functions_equal_host():
    rng = np.random.default_rng(24)
    t = np.concatenate([rng.uniform(-140.0, 140.0, 1 << 19), rng.uniform(-12.0, 12.0, 1 << 19)]).astype(np.float32)
    for fn in (_native.NUM_EXP2_F32, _native.NUM_GELU_F32, _native.NUM_GELU_GRAD_F32):
        got, want = _device_eval(fn, t)
        assert _same_bits(got, want), fn
