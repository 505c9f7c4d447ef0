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
