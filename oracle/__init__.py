"""CPU oracle of the reference simulation semantics — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this package, and only as the checker or the timed CPU baseline.  The
product (cusmc_b200, its CLI and libcsmc.so) never loads it.

liboracle.so is built from oracle/oracle.cpp by cusmc_b200/csrc/Makefile.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from cusmc_b200._native import Query, Result

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `make -f cusmc_b200/csrc/Makefile oracle/liboracle.so`")
        h = ctypes.CDLL(LIB_PATH)
        h.oracle_last_error.restype = ctypes.c_char_p
        h.oracle_run.restype = ctypes.c_int
        h.oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(Query), ctypes.c_uint64,
                                 ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Result),
                                 ctypes.POINTER(ctypes.c_double)]
        h.oracle_trace.restype = ctypes.c_int
        h.oracle_trace.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(Query), ctypes.c_uint64,
                                   ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t,
                                   ctypes.POINTER(ctypes.c_size_t)]
        h.oracle_is_run.restype = ctypes.c_int
        h.oracle_is_run.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(Query), ctypes.c_char_p,
                                    ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.POINTER(ctypes.c_double)]
        h.oracle_is_trace.restype = ctypes.c_int
        h.oracle_is_trace.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(Query), ctypes.c_char_p,
                                      ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                                      ctypes.POINTER(ctypes.c_uint64)]
        h.oracle_mlp_theta.restype = ctypes.c_float
        h.oracle_mlp_theta.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
        h.oracle_mlp_grad.restype = ctypes.c_int
        h.oracle_mlp_grad.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                      ctypes.POINTER(ctypes.c_double)]
        h.oracle_numeric_eval.restype = ctypes.c_int
        h.oracle_numeric_eval.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.c_void_p]
        _lib = h
    return _lib


def run(blob: bytes, query: Query, seed: int, n_runs: int, first_run: int = 0, threads: int = 1,
        digests: bool = False, final_state: bool = False):
    """Simulates runs on the host.  Returns (Result, dict of numpy arrays,
    wall milliseconds of the run loop)."""
    import struct
    n_comps, n_vars = struct.unpack_from("<II", blob, 16)[0], struct.unpack_from("<I", blob, 36)[0]
    flags = np.zeros(n_runs, dtype=np.uint8)
    values = np.zeros(n_runs, dtype=np.float64)
    steps = np.zeros(n_runs, dtype=np.uint32)
    dg = np.zeros(n_runs, dtype=np.uint64) if digests else None
    fs = np.zeros((n_runs, n_comps + n_vars), dtype=np.uint32) if final_state else None
    r = Result()
    ms = ctypes.c_double()
    rc = lib().oracle_run(blob, len(blob), ctypes.byref(query), seed & (2**64 - 1), first_run, n_runs, threads,
                          flags.ctypes.data, values.ctypes.data, steps.ctypes.data,
                          None if dg is None else dg.ctypes.data, None if fs is None else fs.ctypes.data,
                          ctypes.byref(r), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError("oracle: " + lib().oracle_last_error().decode())
    out = {"flags": flags, "values": values, "steps": steps}
    if dg is not None:
        out["digests"] = dg
    if fs is not None:
        out["final_state"] = fs
    return r, out, ms.value


# ---- importance sampling --------------------------------------------------

ROW_DTYPE = np.dtype([("x", "<u2", (16,)), ("a", "<f4"), ("b", "<f4")])  # csmc::MlpRow, 40 bytes


def is_run(blob: bytes, query: Query, params: bytes, seed: int, n_runs: int, first_run: int = 0, threads: int = 0,
           features: bytes | None = None):
    """Runs under the proposal network on the host: dict of per-run flags,
    logw, values, steps; wall milliseconds.  features: a packed feature
    source (cusmc_b200.proposal.pack_features), None for the default."""
    flags = np.zeros(n_runs, dtype=np.uint8)
    logw = np.zeros(n_runs, dtype=np.float64)
    values = np.zeros(n_runs, dtype=np.float64)
    steps = np.zeros(n_runs, dtype=np.uint32)
    ms = ctypes.c_double()
    rc = lib().oracle_is_run(blob, len(blob), ctypes.byref(query), params, features, seed & (2**64 - 1), first_run,
                             n_runs,
                             threads, flags.ctypes.data, logw.ctypes.data, values.ctypes.data, steps.ctypes.data,
                             ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError("oracle: " + lib().oracle_last_error().decode())
    return {"flags": flags, "logw": logw, "values": values, "steps": steps}, ms.value


def is_trace(blob: bytes, query: Query, params: bytes, seed: int, runs, weights, first_run: int = 0,
             cap: int = 1 << 22, features: bytes | None = None) -> np.ndarray:
    """Training rows of the listed runs (four per step, run-list order)."""
    runs = np.ascontiguousarray(runs, dtype=np.uint64)
    weights = np.ascontiguousarray(weights, dtype=np.float32)
    rows = np.zeros(cap, dtype=ROW_DTYPE)
    n = ctypes.c_uint64()
    rc = lib().oracle_is_trace(blob, len(blob), ctypes.byref(query), params, features, seed & (2**64 - 1), first_run,
                               runs.ctypes.data, weights.ctypes.data, len(runs), rows.ctypes.data, cap,
                               ctypes.byref(n))
    if rc != 0:
        raise RuntimeError("oracle: " + lib().oracle_last_error().decode())
    return rows[: n.value].copy()


def mlp_theta(params: bytes, x) -> float:
    x = np.ascontiguousarray(x, dtype=np.float32)
    return float(lib().oracle_mlp_theta(params, x.ctypes.data))


def mlp_grad(params: bytes, rows: np.ndarray):
    """Gradient of sum (b theta - a e^theta) (float32[5313]) and the objective."""
    rows = np.ascontiguousarray(rows)
    g = np.zeros(5313, dtype=np.float32)
    J = ctypes.c_double()
    rc = lib().oracle_mlp_grad(params, rows.ctypes.data, len(rows), g.ctypes.data, ctypes.byref(J))
    if rc != 0:
        raise RuntimeError("oracle: " + lib().oracle_last_error().decode())
    return g, J.value


# ---- numeric primitives -----------------------------------------------------

_NUM_OUT = {0: np.uint32, 1: np.float32, 2: np.float32, 3: np.float64, 4: np.float64, 5: np.float64,
            6: np.float32, 7: np.float32, 8: np.float32, 9: np.uint32}


def numeric(fn: int, a, b=None) -> np.ndarray:
    """Host evaluation of a numeric primitive (csmc_numeric_eval's codes):
    Philox takes counters (n, 4) and keys (n, 2) as uint32 and returns (n, 4)."""
    a = np.ascontiguousarray(a)
    b = None if b is None else np.ascontiguousarray(b)
    n = a.shape[0]
    out = np.zeros((n, 4) if fn in (0, 9) else n, dtype=_NUM_OUT[fn])
    rc = lib().oracle_numeric_eval(fn, a.ctypes.data, None if b is None else b.ctypes.data, n, out.ctypes.data)
    if rc != 0:
        raise RuntimeError("oracle: " + lib().oracle_last_error().decode())
    return out
