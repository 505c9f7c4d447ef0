"""Host-side interface over the C ABI, mirroring the reference's operator
interface for the simulation path.

Reference interface (AndreasHolt/cuSMC) and its counterpart here:

* ``smc(configuration, statistics_Configuration)`` (smc.cuh:14, smc.cu:283)
  -> :func:`smc` with :class:`Configuration` / :class:`StatisticsConfiguration`
  (same fields as main.cuh:33-58); prints the same report.
* ``init_shared_model_state(...)`` (simulation/state/shared_model_state.cuh:219)
  -> :func:`compile_model` + :class:`Network` (upload of the packed network).
* ``run_statistical_model_checking(...)`` (smc.cu:11) plus ``Statistics``
  collection (simulation/statistics.cuh:126-163) -> :meth:`Network.run`
  (device outputs) and :func:`run_host` (host outputs, copies included).

Per-run device buffers are torch CUDA tensors (torch is used for device
memory and streams only); every simulation runs in the sm_100a kernels of
libcsmc.so.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native
from ._native import QUERY_LOCATION, QUERY_VARIABLE, Query, Result, check, lib


@dataclass
class Configuration:
    """main.cuh:33-36."""

    filename: str
    curand_seed: int = 1235


@dataclass
class StatisticsConfiguration:
    """main.cuh:46-58 (``statistics_Configuration``)."""

    simulations: int = 16384
    timeBound: int = 100
    variable_threshhold: int = -1
    variable_id: int = 1
    isMax: bool = True
    isEstimate: bool = True
    loc_query: str = ""


def make_query(kind: int = QUERY_VARIABLE, var_id: int = -1, is_max: bool = True, is_estimate: bool = False,
               threshold: float = 0.0, horizon: float = 100.0, max_steps: int = 0) -> Query:
    q = Query()
    q.kind = kind
    q.var_id = var_id
    q.is_max = 1 if is_max else 0
    q.is_estimate = 1 if is_estimate else 0
    q.threshold = float(threshold)
    q.horizon = float(horizon)
    q.max_steps = int(max_steps)
    return q


def location_query(horizon: float, max_steps: int = 0) -> Query:
    return make_query(QUERY_LOCATION, -1, True, False, 0.0, horizon, max_steps)


def variable_query(var_id: int, horizon: float, threshold: float = 0.0, is_max: bool = True,
                   is_estimate: bool = False, max_steps: int = 0) -> Query:
    return make_query(QUERY_VARIABLE, var_id, is_max, is_estimate, threshold, horizon, max_steps)


def compile_model(path: str, loc_query: str = "", loc_mode: bool = False) -> bytes:
    """Parses a UPPAAL model with the reference's front-end semantics and
    returns the packed network blob."""
    blob = ctypes.c_void_p()
    size = ctypes.c_size_t()
    check(lib().csmc_model_compile(path.encode(), loc_query.encode(), 1 if loc_mode else 0,
                                   ctypes.byref(blob), ctypes.byref(size)))
    try:
        return ctypes.string_at(blob, size.value)
    finally:
        lib().csmc_free(blob)


def dump_model(path: str, loc_query: str = "", loc_mode: bool = False) -> str:
    """Canonical text form of the network as the kernel receives it."""
    text = ctypes.c_void_p()
    check(lib().csmc_model_dump(path.encode(), loc_query.encode(), 1 if loc_mode else 0, ctypes.byref(text)))
    try:
        return ctypes.string_at(text).decode()
    finally:
        lib().csmc_free(text)


def blob_info(blob: bytes) -> dict:
    nv, nc, nl = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    check(lib().csmc_blob_info(blob, len(blob), ctypes.byref(nv), ctypes.byref(nc), ctypes.byref(nl)))
    return {"n_vars": nv.value, "n_comps": nc.value, "n_locs": nl.value}


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


class Network:
    """A packed network resident on the current CUDA device."""

    def __init__(self, blob: bytes):
        self.blob = blob
        self.info = blob_info(blob)
        h = ctypes.c_void_p()
        check(lib().csmc_net_upload(blob, len(blob), ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h:
            lib().csmc_net_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def plan(self) -> tuple[int, int, int]:
        a, b, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check(lib().csmc_plan(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def set_plan(self, family: int, lanes_per_run: int = 32, comps_per_lane: int = 1,
                 threads_per_cta: int = 128) -> None:
        """Selects the kernel family and launch shape (0: lane groups, 1: one
        thread per run, 2: one thread per run with the network in global
        memory)."""
        check(lib().csmc_set_plan(self._h, family, lanes_per_run, comps_per_lane, threads_per_cta))

    def autotune(self, query: Query, seed: int, probe_runs: int) -> Result:
        """Times every feasible launch plan on runs 0..probe_runs-1 and keeps
        the fastest (csmc_autotune); returns the winning probe's result."""
        r = Result()
        check(lib().csmc_autotune(self._h, ctypes.byref(query), seed & (2**64 - 1), probe_runs, ctypes.byref(r)))
        return r

    def run(self, query: Query, seed: int, n_runs: int, first_run: int = 0, flags=None, values=None, steps=None,
            stream: int | None = None) -> Result:
        """Simulates runs on the device; flags/values/steps are optional torch
        CUDA tensors (uint8 / float64 / int32) of at least n_runs entries."""
        r = Result()
        check(lib().csmc_run(self._h, ctypes.byref(query), seed & (2**64 - 1), first_run, n_runs, _ptr(flags),
                             _ptr(values), _ptr(steps), ctypes.byref(r), stream))
        return r

    def run_verify(self, query: Query, seed: int, n_runs: int, first_run: int = 0):
        """Runs the verification variant; returns (Result, dict of numpy arrays)."""
        import torch
        dev = torch.device("cuda")
        C, V = self.info["n_comps"], self.info["n_vars"]
        flags = torch.zeros(n_runs, dtype=torch.uint8, device=dev)
        values = torch.zeros(n_runs, dtype=torch.float64, device=dev)
        steps = torch.zeros(n_runs, dtype=torch.int32, device=dev)
        digests = torch.zeros(n_runs, dtype=torch.int64, device=dev)
        final = torch.zeros(n_runs * (C + V), dtype=torch.int32, device=dev)
        r = Result()
        check(lib().csmc_run_verify(self._h, ctypes.byref(query), seed & (2**64 - 1), first_run, n_runs,
                                    _ptr(flags), _ptr(values), _ptr(steps), _ptr(digests), _ptr(final),
                                    ctypes.byref(r), None))
        out = {
            "flags": flags.cpu().numpy(),
            "values": values.cpu().numpy(),
            "steps": steps.cpu().numpy().view(np.uint32),
            "digests": digests.cpu().numpy().view(np.uint64),
            "final_state": final.cpu().numpy().view(np.uint32).reshape(n_runs, C + V),
        }
        return r, out


class Batch:
    """Many (network, query) jobs simulated by one persistent launch
    (csmc_batch_*).  jobs: list of (Network, Query, seed, n_runs) or
    (Network, Query, seed, n_runs, first_run)."""

    def __init__(self, jobs, verify: bool = False):
        n = len(jobs)
        self.jobs = list(jobs)
        nets = (ctypes.c_void_p * n)(*[j[0]._h for j in jobs])
        qs = (Query * n)(*[j[1] for j in jobs])
        seeds = (ctypes.c_uint64 * n)(*[j[2] & (2**64 - 1) for j in jobs])
        runs = (ctypes.c_uint64 * n)(*[j[3] for j in jobs])
        firsts = (ctypes.c_uint64 * n)(*[(j[4] if len(j) > 4 else 0) for j in jobs])
        h = ctypes.c_void_p()
        check(lib().csmc_batch_create(nets, qs, seeds, firsts, runs, n, 1 if verify else 0, ctypes.byref(h)))
        self._h = h
        self.verify = verify

    def close(self) -> None:
        if self._h:
            lib().csmc_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_plan(self, threads_per_cta: int, ctas_per_sm: int = 0) -> None:
        check(lib().csmc_batch_set_plan(self._h, threads_per_cta, ctas_per_sm))

    def plan(self) -> tuple[int, int]:
        a, b = ctypes.c_int32(), ctypes.c_int32()
        check(lib().csmc_batch_plan(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_group_comps(self, min_comps: int) -> None:
        """Networks of min_comps .. 512 components run one warp per run (0:
        none)."""
        check(lib().csmc_batch_set_group_comps(self._h, min_comps))

    def group_comps(self) -> tuple[int, int]:
        """(warp-per-run threshold, number of jobs it selects)."""
        a, b = ctypes.c_int32(), ctypes.c_int32()
        check(lib().csmc_batch_group_comps(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def autotune(self, probe_fraction: float = 0.05) -> tuple[int, int]:
        a, b = ctypes.c_int32(), ctypes.c_int32()
        check(lib().csmc_batch_autotune(self._h, probe_fraction, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def run(self, use_graph: bool = True, stream: int | None = None) -> list[Result]:
        """Runs the whole batch; one Result per job, in job order."""
        outs = (Result * len(self.jobs))()
        check(lib().csmc_batch_run(self._h, 1 if use_graph else 0, stream, outs))
        return list(outs)

    def outputs(self, job: int) -> dict:
        """Per-run outputs of one job as numpy arrays."""
        net = self.jobs[job][0]
        n = self.jobs[job][3]
        C, V = net.info["n_comps"], net.info["n_vars"]
        flags = np.zeros(n, dtype=np.uint8)
        values = np.zeros(n, dtype=np.float64)
        steps = np.zeros(n, dtype=np.uint32)
        digests = np.zeros(n, dtype=np.uint64) if self.verify else None
        final = np.zeros(n * (C + V), dtype=np.uint32) if self.verify else None
        check(lib().csmc_batch_outputs_host(self._h, job, flags.ctypes.data, values.ctypes.data, steps.ctypes.data,
                                            None if digests is None else digests.ctypes.data,
                                            None if final is None else final.ctypes.data))
        out = {"flags": flags, "values": values, "steps": steps}
        if self.verify:
            out["digests"] = digests
            out["final_state"] = final.reshape(n, C + V)
        return out


def run_host(blob: bytes, query: Query, seed: int, n_runs: int, first_run: int = 0, want_steps: bool = False,
             out: tuple | None = None):
    """Host buffers in and out (upload, kernel, copies back). Returns
    (Result, flags, values, steps-or-None) with numpy arrays.  out: optional
    (flags uint8, values float64, steps uint32 or None) arrays of at least
    n_runs entries to fill instead of new ones."""
    if out is not None:
        flags, values, steps = out
        for a, dt in ((flags, np.uint8), (values, np.float64), (steps, np.uint32)):
            if a is not None and (a.dtype != dt or a.size < n_runs or not a.flags.c_contiguous):
                raise ValueError("run_host: output arrays must be contiguous, of the right type and size")
    else:
        flags = np.empty(n_runs, dtype=np.uint8)
        values = np.empty(n_runs, dtype=np.float64)
        steps = np.empty(n_runs, dtype=np.uint32) if want_steps else None
    r = Result()
    check(lib().csmc_run_host(blob, len(blob), ctypes.byref(query), seed & (2**64 - 1), first_run, n_runs,
                              flags.ctypes.data, values.ctypes.data,
                              None if steps is None else steps.ctypes.data, ctypes.byref(r)))
    return r, flags, values, steps


def smc(conf: Configuration, stat_conf: StatisticsConfiguration) -> None:
    """The reference's ``smc()``: parse, simulate, print the report, update
    ../results5.csv."""
    check(lib().csmc_smc(conf.filename.encode(), int(conf.curand_seed), int(stat_conf.simulations),
                         int(stat_conf.timeBound), int(stat_conf.variable_threshhold), int(stat_conf.variable_id),
                         1 if stat_conf.isMax else 0, 1 if stat_conf.isEstimate else 0,
                         stat_conf.loc_query.encode()))


def parse_query(xml_path: str, formula: str):
    """An UPPAAL formula (Pr[<=T](<> P.loc), Pr[<=T](<> v >= k), E[<=T; N](max: v))
    -> (Query, location name or "", run count or 0)."""
    q = Query()
    loc = ctypes.create_string_buffer(512)
    sims = ctypes.c_uint64()
    check(lib().csmc_query_parse(xml_path.encode(), formula.encode(), ctypes.byref(q), loc, 512, ctypes.byref(sims)))
    return q, loc.value.decode(), sims.value


def smc_ex(model: str, seed: int, sims: int, query: Query, loc_query: str = "", json_path: str | None = None,
           runs_path: str | None = None) -> None:
    """smc() with a full query and optional JSON summary / per-run CSV."""
    check(lib().csmc_smc_ex(model.encode(), int(seed), int(sims), ctypes.byref(query), loc_query.encode(),
                            json_path.encode() if json_path else None, runs_path.encode() if runs_path else None))


def measure_smem_bandwidth() -> tuple[float, float]:
    """Measured shared-memory bandwidth of the current device: (GB/s, mean
    SM clock in MHz during the measurement)."""
    gbs, mhz = ctypes.c_double(), ctypes.c_double()
    check(lib().csmc_measure_smem_bandwidth(ctypes.byref(gbs), ctypes.byref(mhz)))
    return gbs.value, mhz.value


def version() -> str:
    return lib().csmc_version().decode()


__all__ = [
    "Batch", "Configuration", "StatisticsConfiguration", "Network", "Query", "Result", "compile_model", "dump_model",
    "blob_info", "make_query", "measure_smem_bandwidth", "parse_query", "smc_ex", "location_query", "variable_query", "run_host", "smc", "version",
    "QUERY_LOCATION", "QUERY_VARIABLE", "_native",
]
