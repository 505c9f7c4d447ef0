"""ctypes binding of libcsmc.so (the C ABI declared in include/csmc.h).

The shared library is built in-tree by ``make -f cusmc_b200/csrc/Makefile``
(``__graft_entry__.build()`` does this).  Loading fails loudly when it is
missing: there is no Python or CPU fallback for the simulation path.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# CSMC_LIBRARY selects another build of the library (for comparing builds).
LIB_PATH = os.environ.get("CSMC_LIBRARY") or os.path.join(_HERE, "libcsmc.so")

CSMC_OK = 0
CSMC_ERR_ARG = -1
CSMC_ERR_MODEL = -2
CSMC_ERR_CUDA = -3
CSMC_ERR_LIMIT = -4
CSMC_ERR_NODEVICE = -5
CSMC_ERR_TIMEOUT = -6

QUERY_LOCATION = 0
QUERY_VARIABLE = 1

# csmc_numeric_eval function codes (include/csmc.h)
NUM_PHILOX = 0
NUM_EXP_DELAY = 1
NUM_LOG2_F32 = 2
NUM_LOG2_F64 = 3
NUM_EXP2_F64 = 4
NUM_POW_F64 = 5
NUM_EXP2_F32 = 6
NUM_GELU_F32 = 7
NUM_GELU_GRAD_F32 = 8
NUM_PHILOX_STEP = 9


class Query(ctypes.Structure):
    """csmc_query."""

    _fields_ = [
        ("kind", ctypes.c_int32),
        ("var_id", ctypes.c_int32),
        ("is_max", ctypes.c_int32),
        ("is_estimate", ctypes.c_int32),
        ("threshold", ctypes.c_double),
        ("horizon", ctypes.c_double),
        ("max_steps", ctypes.c_uint64),
    ]


class Result(ctypes.Structure):
    """csmc_result."""

    _fields_ = [
        ("runs", ctypes.c_uint64),
        ("hits", ctypes.c_uint64),
        ("steps", ctypes.c_uint64),
        ("capped", ctypes.c_uint64),
        ("sum", ctypes.c_double),
        ("sum_sq", ctypes.c_double),
        ("estimate", ctypes.c_double),
        ("kernel_ms", ctypes.c_double),
        ("lanes_per_run", ctypes.c_int32),
        ("comps_per_lane", ctypes.c_int32),
        ("runs_per_cta", ctypes.c_int32),
        ("family", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class CeConfig(ctypes.Structure):
    """csmc_ce_config."""

    _fields_ = [
        ("rounds", ctypes.c_int32),
        ("adam_steps", ctypes.c_int32),
        ("runs_per_round", ctypes.c_uint64),
        ("max_rows", ctypes.c_uint64),
        ("rho", ctypes.c_double),
        ("lr", ctypes.c_double),
        ("settle", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]


class CeRound(ctypes.Structure):
    """csmc_ce_round."""

    _fields_ = [
        ("round", ctypes.c_int32),
        ("elite", ctypes.c_int32),
        ("rows", ctypes.c_uint64),
        ("level", ctypes.c_double),
        ("j_start", ctypes.c_double),
        ("j_end", ctypes.c_double),
        ("estimate", ctypes.c_double),
        ("hits", ctypes.c_uint64),
        ("capped", ctypes.c_uint64),
        ("mean_steps", ctypes.c_double),
        ("kernel_ms", ctypes.c_double),
        ("run_s", ctypes.c_double),
        ("trace_s", ctypes.c_double),
        ("adam_s", ctypes.c_double),
        ("at_goal", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad"}


class CsmcError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"csmc error {code}: {message}")
        self.code = code


_lib = None

# Every entry point of include/csmc.h with its ctypes signature.
_SIGNATURES = {
    "csmc_last_error": (ctypes.c_char_p, []),
    "csmc_version": (ctypes.c_char_p, []),
    "csmc_model_compile": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]),
    "csmc_model_dump": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "csmc_blob_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    "csmc_free": (None, [ctypes.c_void_p]),
    "csmc_net_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]),
    "csmc_net_free": (None, [ctypes.c_void_p]),
    "csmc_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Query), ctypes.c_uint64, ctypes.c_uint64,
                                ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.POINTER(Result), ctypes.c_void_p]),
    "csmc_run_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(Query), ctypes.c_uint64,
                                     ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.POINTER(Result)]),
    "csmc_run_host_release": (None, []),
    "csmc_run_verify": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Query), ctypes.c_uint64, ctypes.c_uint64,
                                       ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Result), ctypes.c_void_p]),
    "csmc_smc": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]),
    "csmc_smc_ex": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Query), ctypes.c_char_p,
                                   ctypes.c_char_p, ctypes.c_char_p]),
    "csmc_query_parse": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(Query), ctypes.c_char_p,
                                        ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)]),
    "csmc_plan": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                 ctypes.POINTER(ctypes.c_int32)]),
    "csmc_set_plan": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                     ctypes.c_int32]),
    "csmc_run_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(Query),
                                        ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Result), ctypes.c_void_p]),
    "csmc_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Query), ctypes.c_uint64, ctypes.c_uint64,
                                     ctypes.POINTER(Result)]),
    "csmc_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(Query),
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.c_int32, ctypes.c_int32,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "csmc_batch_set_plan": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    "csmc_batch_plan": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                       ctypes.POINTER(ctypes.c_int32)]),
    "csmc_batch_set_group_comps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "csmc_batch_group_comps": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                              ctypes.POINTER(ctypes.c_int32)]),
    "csmc_batch_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "csmc_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.POINTER(Result)]),
    "csmc_batch_results": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Result)]),
    "csmc_batch_outputs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]),
    "csmc_batch_outputs_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "csmc_batch_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32)]),
    "csmc_batch_free": (None, [ctypes.c_void_p]),
    "csmc_is_set_inference": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "csmc_is_set_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "csmc_is_set_features": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]),
    "csmc_is_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Query), ctypes.c_char_p, ctypes.c_uint64,
                                   ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Result), ctypes.c_void_p]),
    "csmc_is_trace": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Query), ctypes.c_char_p, ctypes.c_uint64,
                                     ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "csmc_mlp_forward": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                        ctypes.c_void_p]),
    "csmc_mlp_grad": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "csmc_mlp_adam": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_double, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                     ctypes.c_void_p]),
    "csmc_mlp_rows_merge": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                           ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p]),
    "csmc_ce_select": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                      ctypes.c_double, ctypes.c_int32, ctypes.c_double, ctypes.c_uint64,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)]),
    "csmc_smc_is": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Query),
                                   ctypes.POINTER(CeConfig), ctypes.c_char_p]),
    "csmc_mlp_pack": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "csmc_mlp_init": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_void_p]),
    "csmc_is_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Query), ctypes.c_uint64, ctypes.POINTER(CeConfig),
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(CeRound),
                                     ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "csmc_numeric_eval": (ctypes.c_int, [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    "csmc_measure_smem_bandwidth": (ctypes.c_int, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
}


def lib():
    """Loads libcsmc.so once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -f cusmc_b200/csrc/Makefile` "
            "(the simulation path has no fallback)")
    handle = ctypes.CDLL(LIB_PATH)
    for name, (restype, argtypes) in _SIGNATURES.items():
        fn = getattr(handle, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = handle
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def check(rc: int) -> None:
    if rc != CSMC_OK:
        msg = lib().csmc_last_error()
        raise CsmcError(rc, msg.decode() if msg else "")
