"""Benchmark: runs/s of statistical model checking on the 100-agent SEIR
epidemic network, Pr[<=100](<> R >= 50), 1,000,000 runs per step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload epidemic_100|random_0|mutex_8|mutex_32|mutex_64|mutex_256|batch_64|rare_is|
                              is_kernel|mlp_grad]

The default workload is the epidemic; the others (the small random network
and the Fischer-style mutex at n = 8, 32, 64, 256) use the same measurement
with their own run counts (1e4 and 1e7 runs per step).  batch_64 times 64
random networks in one graph-captured persistent launch against 64
sequential launches; rare_is times learned importance sampling (CE training
included) to a 10%-relative-error interval against plain SMC's rate;
is_kernel times the importance-sampling kernel alone under the trained
proposal, mlp_grad the tensor-core CE gradient on synthetic rows.

A step is one pass of the hot path over one batch: 1e6 independent runs of
the epidemic network (seeded synthetic input: the network comes from
cusmc_b200.netgen.epidemic; every step uses a fresh stretch of the random
stream).  `value` is whole-job runs/s with the network already resident on
the device, timed with CUDA events on the launching stream around the
simulation kernels; `e2e` is the same metric through the host-buffer C-ABI
call csmc_run_host (the network copied to the device, the simulation, the
per-run flags and values copied back into host arrays, all inside the timed
region, after as many untimed warm-up calls as the device-side measurement).  Under torchrun
every rank simulates its own run range (weak scaling, no data-path
collective); times are the max over ranks.

--impl reference times the reference cuSMC binary, built from the reference
sources for sm_100a by oracle/ref/Makefile (oracle/_ref/cusmc_ref_v{8,16,64,512}:
limits raised to that many variables and 8 enabled edges; the smallest build
that holds the network's variables is used), on the same model file and query,
from its own "Time taken" report (kernel + synchronise, smc.cu:234-255), on
rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RUNS_PER_STEP = 1_000_000
SEED = 20241203

# name -> (generator, description); runs per step default to the workload's
# own run count (the epidemic: 1e6)
WORKLOADS = {
    "epidemic_100": (lambda: _netgen().epidemic(n_agents=100, runs=RUNS_PER_STEP),
                     "100-agent SEIR epidemic, Pr[<=100](<> R>=50)"),
    "random_0": (lambda: _netgen().random_network(0, runs=10_000),
                 "random network seed 0: 8 components x 4 locations x 6 edges, 1 clock each, 2 ints, "
                 "Pr[<=100](<> v0>=target)"),
    "mutex_8": (lambda: _netgen().mutex(8), "Fischer-style mutex n=8, Pr[<=200](<> incs>=2)"),
    "mutex_32": (lambda: _netgen().mutex(32), "Fischer-style mutex n=32, Pr[<=200](<> incs>=2)"),
    "mutex_64": (lambda: _netgen().mutex(64), "Fischer-style mutex n=64, Pr[<=200](<> incs>=2)"),
    "mutex_256": (lambda: _netgen().mutex(256), "Fischer-style mutex n=256, Pr[<=200](<> incs>=2)"),
}


def _netgen():
    from cusmc_b200 import netgen
    return netgen


# the rare event of the importance-sampling workload: (T, threshold) with
# goal R > threshold (plain-SMC probability about 1e-6)
IS_RARE = (75, 94)
# CE training of the rare_is workload: up to 12 rounds of 1e4 runs, 40 Adam
# steps per round on at most 1e6 rows, stop once a round's level is the goal
IS_CE = dict(rounds=12, runs_per_round=10_000, adam_steps=40, lr=3e-2, max_rows=1_000_000, settle=1)
IS_CHUNK = 20_000
# the batch workload's run budgets (log-uniform in [1e3, 1e6]) are divided by
# this so that one batch takes seconds (the full budgets take minutes)
BATCH_BUDGET_DIVISOR = 100


def metric_of(name):
    return f"runs/s at 1 B200 ({WORKLOADS[name][1]})"


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def workload_blob(name):
    from cusmc_b200 import api
    w = WORKLOADS[name][0]()
    d = tempfile.mkdtemp(prefix="csmc_bench_")
    path = w.write(os.path.join(d, name + ".xml"))
    blob = api.compile_model(path)
    q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, is_estimate=False)
    return w, path, blob, q


def profile_traffic_per_run(name, family):
    """DRAM bytes (read + write) per run of the simulation kernel the plan
    uses, from the ncu capture summarised in profiles/ (a smaller launch of
    the same kernel and network, scaled by runs): the line
    `dram_bytes_per_run = X` of profiles/<kernel>_<workload>.md."""
    kernel = {4: "coded_kernel", 1: "serial_kernel"}.get(family)
    p = os.path.join(ROOT, "profiles", f"{kernel}_{name}.md")
    if kernel is None or not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            line = line.strip().strip("`")
            if line.startswith("dram_bytes_per_run ="):
                return float(line.split("=")[1])
    return None


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def cpu_baseline(blob, q, budget_s: float = 12.0):
    """The CPU oracle on all host threads, on a bounded sample of the same
    workload (runs from the same stream)."""
    import oracle
    threads = os.cpu_count() or 1
    n = max(threads * 4, 64)
    _, _, ms = oracle.run(blob, q, SEED, n, first_run=0, threads=threads)
    rate = n / (ms / 1000.0)
    n2 = int(min(max(rate * budget_s, n), 200_000))
    r, _, ms2 = oracle.run(blob, q, SEED, n2, first_run=0, threads=threads)
    return {"value": n2 / (ms2 / 1000.0), "unit": "runs/s", "cores": threads, "kind": "port",
            "sample": f"{n2} runs of the same network and query (runs 0..{n2 - 1} of the stream), "
                      f"{ms2 / 1000.0:.1f} s on {threads} host threads"}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from cusmc_b200 import api

    rank, world, local = _env_rank()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    w, path, blob, q = workload_blob(args.workload)
    net = api.Network(blob)
    if args.plan:
        net.set_plan(*[int(x) for x in args.plan.split(",")])
    n = args.runs or w.runs
    dev = torch.device("cuda", local)
    flags = torch.empty(n, dtype=torch.uint8, device=dev)
    values = torch.empty(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev).cuda_stream

    from cusmc_b200 import shard

    def first_run_of(step):
        return shard.first_run(step, rank, world, n)

    for s in range(args.warmup):
        net.run(q, SEED, n, first_run_of(1000 + s), flags=flags, values=values, stream=stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    kernel_ms = []
    hits = 0
    steps_total = 0
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    for s in range(args.steps):
        flush.fill_(float(s))
        ev[s][0].record()
        r = net.run(q, SEED, n, first_run_of(s), flags=flags, values=values, stream=stream)
        ev[s][1].record()
        kernel_ms.append(r.kernel_ms)
        hits += r.hits
        steps_total += r.steps
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_total = sum(step_ms)
    t_kernel = sum(kernel_ms)
    (hits, steps_total), (t_total, t_kernel) = shard.combine([hits, steps_total], [t_total, t_kernel], dev)
    runs_total = n * args.steps * world
    value = runs_total / (t_total / 1000.0)

    # end to end through the host-buffer C-ABI call (rank-local): every step
    # copies the network to the device and the per-run flags and values back
    # into the same host arrays (a caller's reused result buffers)
    h_flags = np.empty(n, dtype=np.uint8)
    h_values = np.empty(n, dtype=np.float64)
    for s in range(args.warmup):
        api.run_host(blob, q, SEED, n, first_run_of(3000 + s), out=(h_flags, h_values, None))
    e2e_ms = []
    e2e_kernel_ms = []
    e2e_sampler = ClockSampler(local)
    e2e_sampler.start()
    for s in range(args.steps):
        t0 = time.perf_counter()
        r_host, _, _, _ = api.run_host(blob, q, SEED, n, first_run_of(2000 + s), out=(h_flags, h_values, None))
        e2e_ms.append((time.perf_counter() - t0) * 1000.0)
        e2e_kernel_ms.append(r_host.kernel_ms)
    e2e_clocks = e2e_sampler.stop()
    e2e_t = sum(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_t], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = t.item()
    e2e_value = runs_total / (e2e_t / 1000.0)

    peak, peak_kind = load_peaks()
    info = api.blob_info(blob)
    n_comps = info["n_comps"]
    plan = net.plan()
    lanes, cpl, rpc = plan
    launch_ms = t_kernel / args.steps
    # algorithmic HBM bytes of one simulation launch: one flag byte and one
    # 8-byte value per run written, the network read once
    alg_bytes = 9 * n + len(blob)
    achieved = alg_bytes / (launch_ms / 1000.0) / 1e9
    traffic_per_run = profile_traffic_per_run(args.workload, r.family)
    # the kernel is bound by instruction issue and shared-memory access, not
    # HBM: one component-step (one component's part in one race) touches
    # 32 B of run state and network records in shared memory
    comp_steps = steps_total * n_comps  # all ranks
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    smem_gbs, smem_mhz = api.measure_smem_bandwidth()
    smem_achieved = 32.0 * comp_steps / world / (t_kernel / 1000.0) / 1e9
    line = {
        "metric": metric_of(args.workload), "value": value, "unit": "runs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 state / f64 expressions", "data": "synthetic (seeded generated network)",
        "config": bench_config(args.workload, n, world),
        "plan": {"family": r.family, "lanes_per_run": lanes, "comps_per_lane": cpl, "runs_per_cta": rpc,
                 "forced": args.plan or None},
        "estimate": hits / runs_total,
        "race_steps_per_run": steps_total / runs_total,
        "component_steps_per_s": comp_steps / (t_total / 1000.0),
        "e2e": {"value": e2e_value, "unit": "runs/s", "h2d_bytes_per_step": len(blob),
                "d2h_bytes_per_step": 9 * n, "ms_per_step": e2e_t / args.steps,
                "kernel_ms_per_step": sum(e2e_kernel_ms) / args.steps, "clocks": e2e_clocks},
        # the binding roofline: 32 B of shared-memory work per component-step
        # over the shared-memory bandwidth measured on this GPU by a streaming
        # 16-byte shared-load kernel (csmc_measure_smem_bandwidth)
        "roofline": {"bound": "smem", "achieved": smem_achieved, "peak": smem_gbs, "unit": "GB/s",
                     "frac": smem_achieved / smem_gbs,
                     "traffic": None if traffic_per_run is None else traffic_per_run * n,
                     "peak_source": f"measured: streaming 16-byte shared-memory loads on every SM "
                                    f"({smem_mhz:.0f} MHz sampled during that kernel)",
                     "bytes_per_component_step": 32, "component_steps_per_launch": comp_steps / world / args.steps,
                     "launch_ms": launch_ms,
                     "traffic_note": "traffic = ncu dram__bytes_read.sum + dram__bytes_write.sum per launch "
                                     "(the kernel's HBM traffic: results only)"},
        "hbm_roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": None if traffic_per_run is None else traffic_per_run * n,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6650 GB/s",
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": launch_ms,
                         "note": "HBM does not bound this kernel (9 B of results per run)"},
        "clocks": clocks,
        "gpu_launches": 2 * args.steps,
        "wall_s": wall,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(blob, q)
    net.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def _netgen_standalone():
    """cusmc_b200/netgen.py loaded as a lone module: the reference arm uses it
    to write the model file and nothing else of this package (no libcsmc)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("csmc_netgen_standalone",
                                                  os.path.join(ROOT, "cusmc_b200", "netgen.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses look their module up by name
    spec.loader.exec_module(mod)
    return mod


def bench_config(name, n, world):
    """The `config` both arms report for workload `name` at n runs per step
    per GPU (identical keys and values, so the two lines describe one
    workload)."""
    return {"workload": f"{name} ({WORKLOADS[name][1]}), {n} runs per step per GPU",
            "runs_per_step_per_gpu": n,
            "l2": "cold between timed steps (our arm: 256 MB L2 flush; reference arm: a fresh process per step)",
            "parallelism": f"runs sharded over {world} GPU(s)"}


# reference arm: warm-up steps are untimed and each is a separate process,
# so they run this many runs each (the timed steps run the full workload)
REF_WARMUP_RUNS = 20_000


def run_reference(args):
    """The reference cuSMC binary (oracle/_ref/cusmc_ref_v*, built from the
    reference sources for sm_100a with raised variable/edge limits) through
    its stock CLI (main.cu:39-110 -> smc.cu:283-491 -> simulation_kernel,
    smc.cu:237), on the same generated model file and query as our arm, at
    the same runs per step.  Each step is one process; the step time is the
    reference's own "Time taken" window (kernel + synchronise,
    smc.cu:234-255).  Nothing of this package is loaded here except the
    stand-alone network generator (no libcsmc)."""
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    netgen = _netgen_standalone()
    gens = {"epidemic_100": lambda: netgen.epidemic(n_agents=100, runs=RUNS_PER_STEP),
            "random_0": lambda: netgen.random_network(0, runs=10_000),
            "mutex_8": lambda: netgen.mutex(8), "mutex_32": lambda: netgen.mutex(32),
            "mutex_64": lambda: netgen.mutex(64), "mutex_256": lambda: netgen.mutex(256)}
    w = gens[args.workload]()
    n = args.runs or w.runs
    # the smallest limits build that holds the network's variables
    variant = next((v for v in (8, 16, 64, 512) if v >= w.n_vars), None)
    binary = os.path.join(ROOT, "oracle", "_ref", f"cusmc_ref_v{variant}")
    if variant is None or not os.path.exists(binary):
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref/cusmc_ref_v{variant} was not built "
                          "(the reference checkout is needed at build time)"}))
        return
    work = tempfile.mkdtemp(prefix="csmc_ref_")
    path = w.write(os.path.join(work, args.workload + ".xml"))
    cwd = os.path.join(work, "run")  # the reference writes ../results5.csv
    os.makedirs(cwd)

    def once(runs, seed):
        cmd = [binary, "-m", path, "-s", str(seed), "-q", str(runs), str(w.horizon), str(w.threshold),
               str(w.var_id), "1", "0", ""]
        out = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=1500)
        ms = None
        result = None
        for line in out.stdout.splitlines():
            if line.startswith("Time taken:") and line.endswith(path) and " ms on file " in line:
                ms = float(line.split()[2])
            if line.startswith("Result:"):
                result = float(line.split()[1])
        if ms is None:
            raise RuntimeError("reference run failed: " + out.stdout[-500:] + out.stderr[-500:])
        return ms, result

    for s in range(args.warmup):
        once(min(n, REF_WARMUP_RUNS), 100 + s)
    sampler = ClockSampler(0)
    sampler.start()
    times, results = [], []
    t_wall = time.perf_counter()
    for s in range(args.steps):
        ms, res = once(n, 1 + s)
        times.append(ms)
        results.append(res)
    wall = time.perf_counter() - t_wall
    clocks = sampler.stop()
    value = n * args.steps / (sum(times) / 1000.0)
    line = {
        "metric": metric_of(args.workload), "value": value, "unit": "runs/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sum(times) / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 state / f64 expressions",
        "data": "synthetic (seeded generated network)", "impl": "reference",
        "config": bench_config(args.workload, n, 1),
        "binary": f"reference cuSMC built from its sources for sm_100a, MAX_VARIABLES={variant}, "
                  "MAX_EDGES_PER_NODE=8 (oracle/ref/Makefile)",
        "warmup_runs_per_step": min(n, REF_WARMUP_RUNS),
        "estimate": statistics.mean(results) if results else None,
        "clocks": clocks, "wall_s": wall,
        # the reference's simulation path is a GPU kernel: it has no CPU
        # implementation, so this describes a GPU run of the reference
        "cpu_baseline": {"value": value, "unit": "runs/s", "cores": 1, "kind": "reference",
                         "where": "GPU (B200): the reference has no CPU implementation of the simulation; "
                                  "one host thread drives its kernel",
                         "sample": f"{n} runs per step, {args.steps} steps, one reference process per step"},
        "e2e": {"value": value, "unit": "runs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _blob_of(w):
    from cusmc_b200 import api
    d = tempfile.mkdtemp(prefix="csmc_bench_")
    return api.compile_model(w.write(os.path.join(d, w.name + ".xml")))


def run_batch(args):
    """64 seeded random networks (2..512 components, 2..8 locations per
    automaton, horizons 50..500, budgets 1e3..1e6 runs divided by
    BATCH_BUDGET_DIVISOR) in one persistent,
    graph-captured launch with an autotuned geometry, against the same jobs as
    64 sequential per-network launches with each network's default plan.
    value = runs/s of the batched launch; `sequential` = runs/s of the 64
    launches."""
    import torch
    from cusmc_b200 import api, netgen
    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    ws = netgen.batch_networks()
    nets = [api.Network(_blob_of(w)) for w in ws]
    jobs = []
    scale = args.batch_divisor or BATCH_BUDGET_DIVISOR
    for i, (w, net) in enumerate(zip(ws, nets)):
        q = api.variable_query(w.var_id, w.horizon, threshold=w.threshold, is_max=True, max_steps=1_000_000)
        jobs.append((net, q, SEED + i, max(10, w.runs // scale), rank * 10 ** 9))
    total = sum(j[3] for j in jobs)
    t_start = time.perf_counter()

    def progress(what):
        print(f"[batch_64] {time.perf_counter() - t_start:8.1f} s  {what}", file=sys.stderr, flush=True)

    progress(f"{len(jobs)} jobs, {total} runs")
    batch = api.Batch(jobs)
    t_tune = time.perf_counter()
    geometry = batch.autotune(probe_fraction=0.02)
    tuned_min = batch.group_comps()[0]
    thresholds = [int(x) for x in str(args.batch_group_comps).split(",")]
    if thresholds[0] >= 0:
        batch.set_group_comps(thresholds[0])
    group = batch.group_comps()
    t_tune = time.perf_counter() - t_tune
    progress(f"autotuned {geometry} (warp-per-run from {tuned_min} components), using {group}")
    for _ in range(args.warmup):
        r0 = batch.run(use_graph=True)
        progress(f"warm-up batch {r0[0].kernel_ms:.1f} ms")
    sampler = ClockSampler(local)
    sampler.start()
    batch_ms = []
    for _ in range(args.steps):
        res = batch.run(use_graph=True)
        batch_ms.append(res[0].kernel_ms)
    clocks = sampler.stop()
    # other warp-per-run thresholds, one timed pass each (results must not change)
    sweep = []
    for m in thresholds[1:]:
        batch.set_group_comps(m)
        r1 = batch.run(use_graph=True)
        same_m = all(a.hits == b.hits and a.steps == b.steps and a.sum == b.sum for a, b in zip(res, r1))
        sweep.append({"min_comps": m, "warp_per_run_jobs": batch.group_comps()[1], "ms": r1[0].kernel_ms,
                      "runs_per_s": total / (r1[0].kernel_ms / 1000.0), "results_identical": same_m})
        progress(f"warp-per-run from {m} components: {r1[0].kernel_ms:.1f} ms")
    # the same jobs as sequential launches
    seq_ms = []
    seq_res = None
    for _ in range(0 if args.batch_no_sequential else max(1, min(args.steps, 2))):
        t = 0.0
        seq_res = []
        for net, q, seed, runs, first in jobs:
            r = net.run(q, seed, runs, first)
            t += r.kernel_ms
            seq_res.append(r)
        seq_ms.append(t)
        progress(f"sequential pass {t:.1f} ms")
    same = all(a.hits == b.hits and a.steps == b.steps for a, b in zip(res, seq_res)) if seq_res else None
    value = total * args.steps / (sum(batch_ms) / 1000.0)
    seq_value = total * len(seq_ms) / (sum(seq_ms) / 1000.0) if seq_ms else None
    line = {"metric": "runs/s at 1 B200 (64 random networks in one launch)", "value": value, "unit": "runs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(batch_ms) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 state / f64 expressions",
            "data": "synthetic (64 seeded generated networks)",
            "config": {"workload": f"batch_64 (random networks, seeds 1000..1063; each run budget / {scale})",
                       "runs_per_step": total,
                       "threads_per_cta": geometry[0], "ctas_per_sm": geometry[1], "graph": True,
                       "warp_per_run_min_comps": group[0], "warp_per_run_jobs": group[1],
                       "autotuned_min_comps": tuned_min},
            "group_sweep": sweep,
            "sequential": ({"value": seq_value, "unit": "runs/s", "ms_per_step": sum(seq_ms) / len(seq_ms)}
                           if seq_ms else None),
            "speedup_vs_sequential": value / seq_value if seq_value else None,
            "results_identical_to_sequential": same,
            "autotune_s": t_tune, "clocks": clocks, "gpu_launches": 2 * args.steps}
    batch.close()
    for n in nets:
        n.close()
    if rank == 0:
        print(json.dumps(line))


def run_rare_is(args):
    """The epidemic with a rare goal (R reaches the threshold within T):
    time to a 10%-relative-error 95% CI, learned importance sampling (CE
    training on the GPU included) against plain SMC at its measured rate."""
    import torch
    from cusmc_b200 import api, netgen, proposal as P
    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    w = netgen.epidemic()
    net = api.Network(_blob_of(w))
    if args.is_tc:
        P.set_inference(net, True)
    if args.is_warp:
        P.set_kernel(net, 3)
    elif args.is_thread:
        P.set_kernel(net, 5)
    T, thr = IS_RARE
    q = api.variable_query(w.var_id, T, threshold=thr, is_max=True)
    ce = dict(IS_CE)
    for key, val in (("rounds", args.ce_rounds), ("runs_per_round", args.ce_runs), ("adam_steps", args.ce_steps)):
        if val:
            ce[key] = val
    if args.ce_rounds:
        ce["settle"] = 0  # exactly the requested number of rounds
    # warm-up outside the timed region: one small CE round and one launch of
    # each simulation kernel load the kernels' modules and allocate the
    # library's device buffers (another seed: nothing carries into the run)
    warm, _ = P.train(net, q, seed=999, rounds=1, runs_per_round=1000, adam_steps=1, lr=ce["lr"],
                      max_rows=100_000)
    P.is_run(net, q, warm.pack(), 999, 4 * 32 * torch.cuda.get_device_properties(local).multi_processor_count,
             1_000_000_000_000)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prop, log = P.train(net, q, seed=1, **ce)
    train_s = time.perf_counter() - t0
    # importance sampling until the 95% CI half-width is 10% of the estimate
    chunk = IS_CHUNK
    s1 = s2 = 0.0
    n = 0
    t1 = time.perf_counter()
    while True:
        r = P.is_run(net, q, prop.pack(), 9, chunk, 2_000_000_000 + n)
        s1 += r.sum
        s2 += r.sum_sq
        n += chunk
        p = s1 / n
        half = 1.96 * math.sqrt(max(s2 / n - p * p, 0.0) / n)
        if (p > 0 and half <= 0.1 * p) or n >= 10_000_000:
            break
    is_s = time.perf_counter() - t1
    # optional fixed-size evaluation of the trained proposal (for example
    # 1e7 weighted runs), outside the timed figure
    evaluation = None
    if args.is_eval_runs:
        t_eval = time.perf_counter()
        p_e, half_e, dev_e = P.estimate(net, q, prop, 19, args.is_eval_runs, first_run=3_000_000_000)
        evaluation = {"runs": args.is_eval_runs, "estimate": p_e, "ci_half": half_e, "device_s": dev_e,
                      "wall_s": time.perf_counter() - t_eval}
    # plain SMC: measured rate, and an estimate on a bounded sample
    plain_n = args.runs or 100_000_000
    hits = 0
    t2 = time.perf_counter()
    done = 0
    while done < plain_n:
        m = min(10_000_000, plain_n - done)
        hits += net.run(q, 13, m, 4_000_000_000 + done).hits
        done += m
    plain_s = time.perf_counter() - t2
    plain_rate = plain_n / plain_s
    p_plain = hits / plain_n
    half_plain = 1.96 * math.sqrt(max(p_plain * (1 - p_plain), 0.0) / plain_n)
    need_plain = 1.96 ** 2 * (1 - p) / (0.01 * p) if p > 0 else float("inf")
    plain_to_10 = need_plain / plain_rate
    line = {"metric": "seconds to a 10%-relative-error 95% CI (learned IS vs plain SMC), epidemic rare event",
            "value": train_s + is_s, "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 network / f32 accumulation / f64 log-weights", "data": "synthetic",
            "config": {"workload": f"epidemic_100, Pr[<={T}](<> R>={thr + 1})", "ce": ce,
                       "sample_chunk": chunk,
                       "inference": "tensor cores (mma.sync bf16)" if args.is_tc else "cuda cores (oracle order)",
                       "kernel": "one thread per run" if r.family == 5 else "one warp per run"},
            "is": {"estimate": p, "ci_half": half, "runs": n, "train_s": train_s, "sample_s": is_s},
            "plain": {"estimate": p_plain, "ci_half": half_plain, "runs": plain_n, "runs_per_s": plain_rate,
                      "runs_for_10pct": need_plain, "seconds_for_10pct": plain_to_10},
            "speedup": plain_to_10 / (train_s + is_s), "is_evaluation": evaluation,
            "agree": abs(p - p_plain) <= half + half_plain,
            "ce_log": log.rounds}
    net.close()
    if rank == 0:
        print(json.dumps(line))


def run_is_kernel(args):
    """The importance-sampling kernel alone: trains the rare_is proposal
    (IS_CE), then times csmc_is_run over --runs runs (default 1e5) per step
    by the CUDA events the call records around its kernel launch.  Kernel
    launches before the timed ones: two per CE round (runs, replay)."""
    import torch
    from cusmc_b200 import api, netgen, proposal as P
    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    w = netgen.epidemic()
    net = api.Network(_blob_of(w))
    if args.is_tc:
        P.set_inference(net, True)
    if args.is_warp:
        P.set_kernel(net, 3)
    elif args.is_thread:
        P.set_kernel(net, 5)
    T, thr = IS_RARE
    q = api.variable_query(w.var_id, T, threshold=thr, is_max=True)
    prop, log = P.train(net, q, seed=1, **IS_CE)
    params = prop.pack()
    n = args.runs or 100_000
    for i in range(args.warmup):
        P.is_run(net, q, params, 9, n, 5_000_000_000 + i * n)
    ms = []
    steps = 0
    family = None
    for i in range(args.steps):
        r = P.is_run(net, q, params, 9, n, 6_000_000_000 + i * n)
        ms.append(r.kernel_ms)
        steps += r.steps
        family = r.family
    net.close()
    t = sum(ms) / 1000.0
    line = {"metric": "runs/s of the importance-sampling kernel under a trained proposal", "value": n * args.steps / t,
            "unit": "runs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 network evaluation / f64 log-weights", "data": "synthetic",
            "config": {"workload": f"epidemic_100, Pr[<={T}](<> R>={thr + 1}), {n} runs per step",
                       "inference": "tensor cores (mma.sync bf16)" if args.is_tc else "cuda cores (oracle order)",
                       "kernel": "one thread per run" if family == 5 else "one warp per run",
                       "ce_rounds": len(log.rounds), "launches_before_timed": 2 * len(log.rounds) + args.warmup},
            "run_steps_per_s": steps / t, "steps_per_run": steps / (n * args.steps)}
    if rank == 0:
        print(json.dumps(line))


def run_mlp_grad(args):
    """The tcgen05 gradient kernel of the proposal network on a seeded
    synthetic row set shaped like the epidemic's training rows (one-hot class,
    S/E/I/R fractions, t/T; a, b weights): rows/s and tensor TFLOP/s.
    FLOP per row counted as the MMAs issue them: forward 2*(16*64 + 64*64),
    back-propagation 2*64*64, weight-gradient GEMM 2*128*96."""
    import torch
    from cusmc_b200 import proposal as P
    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    n = args.runs or 4_000_000
    rng = np.random.default_rng(SEED)
    x = np.zeros((n, 16), np.float32)
    x[np.arange(n), rng.integers(0, 4, n)] = 1.0
    frac = rng.dirichlet([4, 1, 1, 4], n).astype(np.float32)
    x[:, 5:9] = frac
    x[:, 9] = rng.uniform(0, 1, n)
    rows = np.zeros(n, dtype=np.dtype([("x", "<u2", (16,)), ("a", "<f4"), ("b", "<f4")]))
    rows["x"] = P.f32_to_bf16_bits(x.ravel()).reshape(n, 16)
    rows["a"] = rng.exponential(1e-3, n).astype(np.float32)
    rows["b"] = (rng.uniform(0, 1, n) < 0.25).astype(np.float32) * 1e-3
    d_rows = torch.from_numpy(rows.view(np.uint8).copy()).cuda()
    prop = P.Proposal.init(1)
    prop.w3 = (rng.standard_normal(64) * 0.05).astype(np.float32)
    params = prop.pack()
    for _ in range(args.warmup):
        P.mlp_grad(params, d_rows, n)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    for _ in range(args.steps):
        P.mlp_grad(params, d_rows, n)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    flop_row = 2 * (16 * 64 + 64 * 64) + 2 * 64 * 64 + 2 * 128 * 96
    peak = 1672.1
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peak = json.load(open(pk)).get("bf16_tflops", peak)
    tflops = flop_row * n / (ms / 1000.0) / 1e12
    line = {"metric": "rows/s of the tensor-core CE gradient (proposal network)", "value": n / (ms / 1000.0),
            "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 operands / f32 accumulation", "data": "synthetic rows (seeded)",
            "config": {"workload": f"mlp_grad, {n} rows", "flop_per_row": flop_row},
            "roofline": {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s",
                         "frac": tflops / peak, "peak_source": "MEASURED_PEAKS.json bf16_tflops"
                         if os.path.exists(pk) else "fallback"},
            "note": "time per call includes the parameter upload, the device reduction of the per-CTA partial "
                    "sums and the copy of the gradient to the host"}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-oracle baseline")
    ap.add_argument("--runs", type=int, default=0,
                    help="runs per step per GPU (default: the workload's run count, 1e6 for the epidemic; "
                         "smaller values are for profiling captures)")
    ap.add_argument("--is-eval-runs", type=int, default=0,
                    help="rare_is: also evaluate the trained proposal on this many weighted runs (e.g. 10000000)")
    ap.add_argument("--ce-rounds", type=int, default=0,
                    help="rare_is: exactly this many CE rounds (default: IS_CE, stopping once settled)")
    ap.add_argument("--ce-runs", type=int, default=0, help="rare_is: runs per CE round (default: IS_CE)")
    ap.add_argument("--ce-steps", type=int, default=0, help="rare_is: Adam steps per CE round (default: IS_CE)")
    ap.add_argument("--plan", default="",
                    help="single-network workloads: launch plan FAMILY,LANES,COMPS_PER_LANE,THREADS_PER_CTA "
                         "(csmc_set_plan; default: the library's choice); the e2e leg keeps the default plan")
    ap.add_argument("--is-warp", action="store_true",
                    help="rare_is / is_kernel: runs under the proposal one warp per run (the thread-per-run "
                         "kernel is the default where the network qualifies)")
    ap.add_argument("--is-thread", action="store_true",
                    help="rare_is / is_kernel: runs under the proposal one thread per run at every launch size "
                         "(the default takes one warp per run below 48 runs per SM on the epidemic)")
    ap.add_argument("--is-tc", action="store_true",
                    help="rare_is / is_kernel: theta by warp-level tensor-core MMAs instead of the CUDA-core "
                         "evaluation in the oracle's order")
    ap.add_argument("--batch-group-comps", default="-1",
                    help="batch_64: networks with at least this many components run one warp per run "
                         "(0: none; -1, the default: the autotuner's choice); further comma-separated "
                         "thresholds are each timed once more and reported under group_sweep")
    ap.add_argument("--batch-no-sequential", action="store_true",
                    help="batch_64: skip the pass of 64 sequential launches")
    ap.add_argument("--batch-divisor", type=int, default=0,
                    help="batch_64: divide every job's run budget by this (default BATCH_BUDGET_DIVISOR)")
    ap.add_argument("--workload", default="epidemic_100", choices=sorted(WORKLOADS) + ["batch_64", "rare_is", "is_kernel", "mlp_grad"],
                    help="network and query (default: the 100-agent epidemic)")
    args = ap.parse_args()
    if args.workload == "batch_64" and args.impl == "ours":
        return run_batch(args)
    if args.workload == "rare_is" and args.impl == "ours":
        return run_rare_is(args)
    if args.workload == "mlp_grad" and args.impl == "ours":
        return run_mlp_grad(args)
    if args.workload == "is_kernel" and args.impl == "ours":
        return run_is_kernel(args)
    if args.workload in ("batch_64", "rare_is", "is_kernel", "mlp_grad"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference simulates one model per process and has "
                          "no importance sampling; this workload has no reference arm"}))
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
