"""Learned importance sampling: the proposal network, its parameter block,
and the cross-entropy (CE) training loop.

The proposal multiplies every exponential rate by exp(theta), theta =
MLP(features) (cusmc_b200/csrc/include/csmc_mlp.h has the feature map and
the exact arithmetic).  Runs under the proposal carry their log-likelihood
ratio w.r.t. the nominal model, so ``flag * exp(logw)`` averages to the
goal probability whatever the network; training only lowers the variance.

CE training (multi-level, Rubinstein's method): each round simulates runs
under the current proposal, takes as elite the runs whose tracked value
reaches the round's level gamma = min(goal, (1-rho)-quantile of the tracked
values), weights each elite run by its likelihood ratio, replays the elite
runs on the GPU into training rows (four per step: features, a, b), and
takes Adam steps on J = sum (b theta - a e^theta), the weighted
log-likelihood of the elite paths under the proposal up to a constant; the
gradient of J comes from the tensor-core kernel, and a round's Adam steps
run on the device (csmc_mlp_adam).
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from ._native import Query, Result, check, lib

HID, IN = 64, 16
GRAD_FLOATS = HID * IN + HID + HID * HID + HID + HID + 1
ROW_BYTES = 40
PARAM_BYTES = 11024
THETA_MAX = 4.0


def f32_to_bf16_bits(a: np.ndarray) -> np.ndarray:
    """Round to nearest even, as f_to_bf16 in csmc_mlp.h."""
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    nan = (b & 0x7FFFFFFF) > 0x7F800000
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)
    r[nan] = ((b[nan] >> 16) | 0x40).astype(np.uint16)
    return r


def bf16_bits_to_f32(h: np.ndarray) -> np.ndarray:
    return (np.asarray(h, dtype=np.uint32) << 16).view(np.float32)


@dataclass
class Proposal:
    """FP32 master parameters; pack() gives the BF16 parameter block."""

    w1: np.ndarray
    b1: np.ndarray
    w2: np.ndarray
    b2: np.ndarray
    w3: np.ndarray
    b3: float = 0.0

    @staticmethod
    def init(seed: int = 0, scale: float = 1.0) -> "Proposal":
        """He-style random hidden layers, zero output layer: theta = 0, the
        proposal starts as the nominal model."""
        rng = np.random.default_rng(seed)
        w1 = (rng.standard_normal((HID, IN)) * math.sqrt(2.0 / 10) * scale).astype(np.float32)
        w1[:, 10:] = 0.0
        w2 = (rng.standard_normal((HID, HID)) * math.sqrt(2.0 / HID) * scale).astype(np.float32)
        return Proposal(w1, np.zeros(HID, np.float32), w2, np.zeros(HID, np.float32), np.zeros(HID, np.float32), 0.0)

    def vector(self) -> np.ndarray:
        return np.concatenate([self.w1.ravel(), self.b1, self.w2.ravel(), self.b2, self.w3,
                               np.array([self.b3], np.float32)]).astype(np.float32)

    @staticmethod
    def from_vector(v: np.ndarray) -> "Proposal":
        v = np.asarray(v, dtype=np.float32)
        o = 0
        w1 = v[o:o + HID * IN].reshape(HID, IN).copy(); o += HID * IN
        b1 = v[o:o + HID].copy(); o += HID
        w2 = v[o:o + HID * HID].reshape(HID, HID).copy(); o += HID * HID
        b2 = v[o:o + HID].copy(); o += HID
        w3 = v[o:o + HID].copy(); o += HID
        return Proposal(w1, b1, w2, b2, w3, float(v[o]))

    def pack(self) -> bytes:
        """csmc::MlpParams: w1 (BF16), b1, w2 (BF16), b2, w3, b3, pad."""
        out = bytearray()
        out += f32_to_bf16_bits(self.w1).tobytes()
        out += np.asarray(self.b1, np.float32).tobytes()
        out += f32_to_bf16_bits(self.w2).tobytes()
        out += np.asarray(self.b2, np.float32).tobytes()
        out += np.asarray(self.w3, np.float32).tobytes()
        out += np.array([self.b3, 0, 0, 0], np.float32).tobytes()
        assert len(out) == PARAM_BYTES
        return bytes(out)


class AdamState:
    """Adam's moments and step count across CE rounds (the steps run on the
    device: adam_run)."""

    def __init__(self, n: int = GRAD_FLOATS):
        self.m = np.zeros(n, np.float64)
        self.v = np.zeros(n, np.float64)
        self.t = 0


def adam_run(rows, n_rows: int, steps: int, lr: float, x: np.ndarray, state: AdamState, stream=None):
    """csmc_mlp_adam: `steps` Adam ascent steps on J over n_rows device rows
    (a torch CUDA tensor), on the device; x (FP32 master vector) and state
    are updated in place.  Returns J at the first and the last step."""
    assert x.dtype == np.float32 and x.size == GRAD_FLOATS and x.flags.c_contiguous
    t = ctypes.c_int32(state.t)
    j0, j1 = ctypes.c_double(), ctypes.c_double()
    check(lib().csmc_mlp_adam(_ptr(rows), n_rows, steps, lr, x.ctypes.data, state.m.ctypes.data,
                              state.v.ctypes.data, ctypes.byref(t), ctypes.byref(j0), ctypes.byref(j1), stream))
    state.t = t.value
    return j0.value, j1.value


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def set_inference(net, tensor_cores: bool) -> None:
    """Warp-level tensor-core evaluation of the proposal, or the CUDA-core one
    (the default: faster for the four rows a step evaluates) that reproduces
    the CPU oracle bit for bit."""
    check(lib().csmc_is_set_inference(net._h, 1 if tensor_cores else 0))


def set_kernel(net, family: int) -> None:
    """Kernel of runs under the proposal: 0 = one thread per run where the
    network qualifies and the launch has at least 48 runs per SM (128 when a
    location is outside the tilt groups; else one warp per run), 3 = always
    one warp per run, 5 = one thread per run
    wherever the network qualifies.  All give the same runs bit for bit."""
    check(lib().csmc_is_set_kernel(net._h, family))


def set_features(net, count_vars=None, scales=None, clock_var: int = -1) -> None:
    """The network's feature source (csmc_is_set_features): count_vars (4
    variable ids, -1 unused) feed features 5..8 times scales; clock_var
    feeds feature 4.  No arguments: the default (variables 0..3 over the
    component count, no clock)."""
    cv = None if count_vars is None else (ctypes.c_int32 * 4)(*count_vars)
    sc = None if scales is None else (ctypes.c_float * 4)(*scales)
    check(lib().csmc_is_set_features(net._h, cv, sc, int(clock_var)))


def pack_features(n_vars: int, n_comps: int, count_vars=None, scales=None, clock_var: int = -1) -> bytes:
    """The same feature source packed as csmc::MlpFeatures (for the CPU
    oracle's is_run / is_trace)."""
    var = list(count_vars) if count_vars is not None else [i if i < n_vars else -1 for i in range(4)]
    inv_c = np.float32(1.0) / np.float32(n_comps)
    sc = list(scales) if scales is not None else [inv_c] * 4
    return (np.array(var, np.int32).tobytes() + np.array(sc, np.float32).tobytes() +
            np.array([clock_var, 0, 0, 0], np.int32).tobytes())


def is_run(net, query: Query, params: bytes, seed: int, n_runs: int, first_run: int = 0, flags=None, logw=None,
           values=None, steps=None, stream=None) -> Result:
    """csmc_is_run on a Network; per-run outputs are optional torch CUDA tensors."""
    r = Result()
    check(lib().csmc_is_run(net._h, ctypes.byref(query), params, seed & (2**64 - 1), first_run, n_runs,
                            _ptr(flags), _ptr(logw), _ptr(values), _ptr(steps), ctypes.byref(r), stream))
    return r


def is_trace(net, query: Query, params: bytes, seed: int, runs, weights, row_offset, rows, first_run: int = 0,
             stream=None) -> None:
    """csmc_is_trace: runs/weights/row_offset/rows are torch CUDA tensors
    (rows: a byte buffer of whole 40-byte rows, its size the row capacity)."""
    check(lib().csmc_is_trace(net._h, ctypes.byref(query), params, seed & (2**64 - 1), first_run, _ptr(runs),
                              _ptr(weights), _ptr(row_offset), len(runs), _ptr(rows),
                              rows.numel() * rows.element_size() // ROW_BYTES, stream))


def mlp_forward(params: bytes, rows, n_rows: int, theta, stream=None) -> None:
    check(lib().csmc_mlp_forward(params, _ptr(rows), n_rows, _ptr(theta), stream))


def merge_rows(rows, row_offset, n_list: int, n_rows: int, out, stream=None) -> int:
    """csmc_mlp_rows_merge: rows, row_offset (the replay's per-run first
    rows) and out are torch CUDA tensors; returns the merged row count."""
    n = ctypes.c_uint64()
    check(lib().csmc_mlp_rows_merge(_ptr(rows), _ptr(row_offset), n_list, n_rows, _ptr(out), ctypes.byref(n),
                                    stream))
    return n.value


def mlp_grad(params: bytes, rows, n_rows: int, stream=None):
    g = np.zeros(GRAD_FLOATS, np.float32)
    J = ctypes.c_double()
    check(lib().csmc_mlp_grad(params, _ptr(rows), n_rows, g.ctypes.data, ctypes.byref(J), stream))
    return g, J.value


@dataclass
class TrainLog:
    rounds: list = field(default_factory=list)


def estimate(net, query: Query, proposal: Proposal | None, seed: int, n_runs: int, first_run: int = 0,
             chunk: int = 2_000_000):
    """Importance-sampling (or, with proposal None, plain) estimate of the
    query's probability: (p, half-width of the 95% CI, device seconds)."""
    import torch  # noqa: F401  (device buffers of the plain path)
    s1 = s2 = 0.0
    dev_s = 0.0
    done = 0
    params = (proposal or Proposal.init()).pack() if proposal is not None else None
    while done < n_runs:
        n = min(chunk, n_runs - done)
        if proposal is None:
            r = net.run(query, seed, n, first_run + done)
            s1 += r.hits
            s2 += r.hits
        else:
            r = is_run(net, query, params, seed, n, first_run + done)
            s1 += r.sum
            s2 += r.sum_sq
        dev_s += r.kernel_ms / 1000.0
        done += n
    p = s1 / n_runs
    var = max(s2 / n_runs - p * p, 0.0)
    half = 1.96 * math.sqrt(var / n_runs)
    return p, half, dev_s


@dataclass
class Elite:
    """One CE round's training set: the level, the elite runs (indices into
    the round), their normalised CE weights (float32), the first row of each
    run's block in the row buffer (four rows per step) and the row count."""

    level: float
    runs: np.ndarray
    weights: np.ndarray
    row_offset: np.ndarray
    n_rows: int
    at_goal: bool


def select_elite(values: np.ndarray, logw: np.ndarray, steps: np.ndarray, threshold: float, is_max: bool = True,
                 rho: float = 0.1, max_rows: int = 40_000_000) -> Elite:
    """Multi-level CE selection for the goal value > threshold (max query) or
    value < threshold (min query), by the library's host routine
    csmc_ce_select (the C++ training loop uses the same one): the level is
    the (1 - rho)-quantile of the runs' scores (the value, negated for a min
    query; linear interpolation between order statistics), capped at the
    goal; the elite are the runs at or beyond the level (strictly beyond the
    goal once the level reaches it), weighted by their likelihood ratios.
    Runs are kept heaviest first while their rows (4 per step) fit in
    max_rows, and at least one run is kept."""
    values = np.ascontiguousarray(values, np.float64)
    logw = np.ascontiguousarray(logw, np.float64)
    steps = np.ascontiguousarray(steps, np.uint32)
    n = len(values)
    elite = np.zeros(n, np.uint64)
    weights = np.zeros(n, np.float32)
    offs = np.zeros(n, np.uint64)
    ne, nr, lev, at = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_double(), ctypes.c_int32()
    check(lib().csmc_ce_select(values.ctypes.data, logw.ctypes.data, steps.ctypes.data, n, float(threshold),
                               1 if is_max else 0, float(rho), int(max_rows), elite.ctypes.data, weights.ctypes.data,
                               offs.ctypes.data, ctypes.byref(ne), ctypes.byref(nr), ctypes.byref(lev),
                               ctypes.byref(at)))
    k = ne.value
    return Elite(lev.value, elite[:k].astype(np.int64), weights[:k].copy(), offs[:k].copy(), int(nr.value),
                 bool(at.value))


def init_c(seed: int = 0) -> "Proposal":
    """The library's initial proposal (csmc_mlp_init; what the CLI trains from)."""
    v = np.zeros(GRAD_FLOATS, np.float32)
    check(lib().csmc_mlp_init(seed & (2**64 - 1), v.ctypes.data))
    return Proposal.from_vector(v)


def train_c(net, query: Query, seed: int = 1, init: "Proposal | None" = None, rounds: int = 10,
            runs_per_round: int = 100_000, rho: float = 0.1, adam_steps: int = 30, lr: float = 3e-3,
            max_rows: int = 40_000_000, settle: int = 0):
    """CE training through the C ABI (csmc_is_train): the same method as
    train(), run by the library.  Returns (Proposal, list of round dicts)."""
    from ._native import CeConfig, CeRound
    x0 = (init or Proposal.init(0)).vector()
    cfg = CeConfig(rounds=rounds, adam_steps=adam_steps, runs_per_round=runs_per_round, max_rows=max_rows, rho=rho,
                   lr=lr, settle=settle)
    out = np.zeros(GRAD_FLOATS, np.float32)
    log = (CeRound * rounds)()
    done = ctypes.c_int32()
    check(lib().csmc_is_train(net._h, ctypes.byref(query), seed & (2**64 - 1), ctypes.byref(cfg), x0.ctypes.data,
                              out.ctypes.data, None, log, rounds, ctypes.byref(done)))
    return Proposal.from_vector(out), [log[i].as_dict() for i in range(done.value)]


def train(net, query: Query, seed: int = 1, rounds: int = 10, runs_per_round: int = 100_000, rho: float = 0.1,
          adam_steps: int = 30, lr: float = 3e-3, init_seed: int = 0, max_rows: int = 40_000_000,
          settle: int = 0, verbose: bool = False):
    """CE training of the proposal on the GPU.  The goal is the query's
    threshold event (tracked value > threshold for a max query, < threshold
    for a min query; a location query has no value to rank runs by and is
    refused).  With settle > 0 training stops after that many rounds whose
    level was the goal itself (at least rho of the round's runs reached it).
    Returns (Proposal, TrainLog); each round's entry has its level, elite
    count, rows, J before and after the Adam steps, and the seconds spent
    simulating, replaying and in the gradient steps."""
    import torch
    if query.kind != 1:
        raise ValueError("CE training needs a variable query (the tracked value ranks the runs)")
    dev = torch.device("cuda")
    prop = Proposal.init(init_seed)
    x = prop.vector()
    opt = AdamState(x.size)
    log = TrainLog()
    n = runs_per_round
    flags = torch.empty(n, dtype=torch.uint8, device=dev)
    logw = torch.empty(n, dtype=torch.float64, device=dev)
    values = torch.empty(n, dtype=torch.float64, device=dev)
    steps = torch.empty(n, dtype=torch.int32, device=dev)
    at_goal = 0
    for k in range(rounds):
        t0 = time.perf_counter()
        params = prop.pack()
        first = (k + 1) * 10_000_000  # each round uses fresh runs of the stream
        res = is_run(net, query, params, seed, n, first, flags=flags, logw=logw, values=values, steps=steps)
        sel = select_elite(values.cpu().numpy(), logw.cpu().numpy(), steps.cpu().numpy().view(np.uint32),
                           query.threshold, bool(query.is_max), rho, max_rows)
        elite, n_rows = sel.runs, sel.n_rows
        rows = torch.empty(n_rows * ROW_BYTES, dtype=torch.uint8, device=dev)
        t_runs = torch.from_numpy(elite.astype(np.uint64).view(np.int64)).to(dev)
        t_w = torch.from_numpy(sel.weights).to(dev)
        t_off = torch.from_numpy(sel.row_offset.view(np.int64)).to(dev)
        t1 = time.perf_counter()
        is_trace(net, query, params, seed, t_runs, t_w, t_off, rows, first)
        # rows of equal features on consecutive steps summed (J unchanged)
        merged = torch.empty_like(rows)
        m_rows = merge_rows(rows, t_off, len(elite), n_rows, merged)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        x = np.array(x, dtype=np.float32, copy=True)
        J0, J = adam_run(merged, m_rows, adam_steps, lr, x, opt)
        prop = Proposal.from_vector(x)
        t3 = time.perf_counter()
        hit_est = float(res.estimate)
        entry = {"round": k, "level": sel.level, "elite": int(len(elite)), "rows": n_rows, "merged_rows": m_rows,
                 "J_start": J0, "J_end": J,
                 "estimate": hit_est, "hits": int(res.hits), "mean_steps": res.steps / max(res.runs, 1),
                 "capped": int(res.capped), "kernel_ms": res.kernel_ms, "run_s": t1 - t0, "trace_s": t2 - t1,
                 "adam_s": t3 - t2, "seconds": t3 - t0}
        log.rounds.append(entry)
        if verbose:
            print(entry, flush=True)
        del rows, merged
        at_goal = at_goal + 1 if sel.at_goal else 0
        if settle and at_goal >= settle:
            break
    return prop, log
