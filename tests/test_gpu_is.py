"""Learned importance sampling on the GPU, checked against the CPU oracle.

* Runs under the proposal (csmc_is_run, CUDA-core evaluation of theta) are
  bit-identical to the oracle's: flags, step counts, tracked values and the
  FP64 log-likelihood ratios; replayed training rows (csmc_is_trace) are
  byte-identical to the oracle's.
* With the tensor-core evaluation of theta (the default), runs follow the
  same paths as the exact evaluation except where a race is decided within
  theta's rounding (a small fraction of runs), their log-likelihood ratios
  agree closely, and replay reproduces the tensor-core runs' own paths.
* The tcgen05 forward pass agrees with the oracle's theta within 1e-2
  (tensor-core accumulation order and BF16 re-rounding of the first hidden
  layer), and the tcgen05 gradient of the CE objective agrees with the
  oracle's gradient block by block within 2% (relative L2 norm).
* CE training on the GPU lowers the relative error of the estimate of a rare
  event, and the trained estimate agrees with plain SMC.
"""
import math
import os
import tempfile

import numpy as np
import pytest

import oracle
from cusmc_b200 import api, netgen, proposal as P

pytestmark = pytest.mark.gpu


def _blob(w):
    with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
        f.write(w.xml)
        path = f.name
    try:
        return api.compile_model(path)
    finally:
        os.unlink(path)


def _random_proposal(seed, out_scale=0.3):
    p = P.Proposal.init(seed)
    rng = np.random.default_rng(seed + 100)
    p.w3 = (rng.standard_normal(64) * out_scale / 8).astype(np.float32)
    p.b3 = 0.1
    return p


def _tilt_mix(n_comps=24):
    """Components of four exponential locations in a cycle whose rates come
    from four shared literals rotated by component, so every rate appears in
    every location class: 16 (race class, location class) pairs, more than
    the six tilt groups (the rest take the descriptor path).  Leaving L3
    broadcasts `go`, which moves receivers in L1 to L2 (L1 has two edges, so
    slot masks are kept); counters v0..v3 feed the proposal's features."""
    rates = ["0.3", "0.7", "1.1", "1.9"]
    d = netgen._Doc("int v0 = 0;\nint v1 = 0;\nint v2 = 0;\nint v3 = 0;\nbroadcast chan go;")
    for c in range(n_comps):
        ids = [d.new_id() for _ in range(4)]
        locs = [(ids[i], f"L{i}", [("exponentialrate", rates[(i + c) % 4])]) for i in range(4)]
        trans = [
            (ids[0], ids[1], [("assignment", "v1 = v1 + 1")]),
            (ids[1], ids[2], [("assignment", "v2 = v2 + 1")]),
            (ids[1], ids[2], [("synchronisation", "go?")]),
            (ids[2], ids[3], [("assignment", "v3 = v3 + 1")]),
            (ids[3], ids[0], [("synchronisation", "go!"), ("assignment", "v0 = v0 + 1")]),
        ]
        d.template(f"M{c}", "", locs, ids[0], trans)
    return netgen.Workload("tilt_mix", d.finish(), var_id=0, threshold=46, horizon=15, runs=1000, n_vars=4)


CASES = {
    "tilt_mix": lambda: (_tilt_mix(), None, None),
    "epidemic": lambda: (netgen.epidemic(), 100, 49),
    # 160 components: lanes 0..7 of the warp draw two Philox blocks each, so
    # their partial sums span two blocks (the warp order of csmc_mlp.h)
    "epidemic_160": lambda: (netgen.epidemic(n_agents=160), 60, 79),
    "random": lambda: (netgen.random_network(3), None, None),
    "mutex": lambda: (netgen.mutex(8), None, None),
}


# networks with race classes: csmc_is_set_kernel(5) simulates them one
# thread per run (family 5) at any launch size; 3 forces one warp per run
THREAD_CASES = {"epidemic", "epidemic_160", "mutex", "tilt_mix"}


@pytest.mark.parametrize("kernel", [5, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_is_runs_match_the_oracle(name, kernel):
    import torch
    w, T, thr = CASES[name]()
    blob = _blob(w)
    q = api.variable_query(w.var_id, T or w.horizon, threshold=thr if thr is not None else w.threshold,
                           is_max=True, max_steps=100_000)
    params = _random_proposal(3).pack()
    n = 512
    net = api.Network(blob)
    P.set_inference(net, False)
    P.set_kernel(net, kernel)
    try:
        dev = torch.device("cuda")
        flags = torch.zeros(n, dtype=torch.uint8, device=dev)
        logw = torch.zeros(n, dtype=torch.float64, device=dev)
        values = torch.zeros(n, dtype=torch.float64, device=dev)
        steps = torch.zeros(n, dtype=torch.int32, device=dev)
        r = P.is_run(net, q, params, 17, n, 40, flags=flags, logw=logw, values=values, steps=steps)
    finally:
        net.close()
    assert r.family == (5 if kernel == 5 and name in THREAD_CASES else 3)
    cpu, _ = oracle.is_run(blob, q, params, 17, n, 40)
    assert np.array_equal(flags.cpu().numpy(), cpu["flags"])
    assert np.array_equal(steps.cpu().numpy().view(np.uint32), cpu["steps"])
    assert np.array_equal(values.cpu().numpy().view(np.uint64), cpu["values"].view(np.uint64))
    assert np.array_equal(logw.cpu().numpy().view(np.uint64), cpu["logw"].view(np.uint64))
    wv = cpu["flags"] * np.exp(cpu["logw"])
    assert r.sum == pytest.approx(wv.sum(), rel=1e-12, abs=1e-300)


def test_theta_cache_keeps_runs_exact_across_launches():
    """The thread-per-run kernel's device-wide theta cache is keyed by the
    feature vector within one parameter block: launches with proposal A, then
    B, then A again (a new generation: A's old entries are not reused), and
    two launches in a row with the same block (the second reads entries the
    first wrote), all equal the oracle's runs bit for bit."""
    import torch
    w = netgen.epidemic()
    blob = _blob(w)
    q = api.variable_query(w.var_id, 100, threshold=49, is_max=True, max_steps=100_000)
    pa, pb = _random_proposal(4).pack(), _random_proposal(5).pack()
    n = 1024
    net = api.Network(blob)
    P.set_inference(net, False)
    P.set_kernel(net, 5)
    try:
        dev = torch.device("cuda")
        for params, first in ((pa, 0), (pb, 0), (pa, 0), (pa, 5000)):
            logw = torch.zeros(n, dtype=torch.float64, device=dev)
            steps = torch.zeros(n, dtype=torch.int32, device=dev)
            r = P.is_run(net, q, params, 23, n, first, logw=logw, steps=steps)
            assert r.family == 5
            cpu, _ = oracle.is_run(blob, q, params, 23, n, first)
            assert np.array_equal(steps.cpu().numpy().view(np.uint32), cpu["steps"])
            assert np.array_equal(logw.cpu().numpy().view(np.uint64), cpu["logw"].view(np.uint64))
    finally:
        net.close()


def test_launch_size_picks_the_kernel_and_keeps_the_runs():
    """csmc_is_run's default: one warp per run below 48 runs per SM on a
    network whose locations are all in tilt groups (the epidemic), one
    thread per run above, in CTAs of 128 threads and, from 576 runs per SM,
    of 384; the runs they share are the same bits."""
    import torch
    w = netgen.epidemic()
    blob = _blob(w)
    q = api.variable_query(w.var_id, 100, threshold=49, is_max=True, max_steps=100_000)
    params = _random_proposal(6).pack()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    huge, big, small = 576 * sms + 1000, 48 * sms + 1000, 2000
    net = api.Network(blob)
    P.set_inference(net, False)
    try:
        dev = torch.device("cuda")
        out = {}
        for n in (huge, big, small):
            logw = torch.zeros(n, dtype=torch.float64, device=dev)
            steps = torch.zeros(n, dtype=torch.int32, device=dev)
            r = P.is_run(net, q, params, 31, n, 100, logw=logw, steps=steps)
            out[n] = (r.family, logw.cpu().numpy(), steps.cpu().numpy(), r.runs_per_cta)
    finally:
        net.close()
    assert out[huge][0] == 5 and out[huge][3] == 384
    assert out[big][0] == 5 and out[big][3] in (32, 64, 128)
    assert out[small][0] == 3
    for n in (huge, big):
        assert np.array_equal(out[n][1][:small].view(np.uint64), out[small][1].view(np.uint64))
        assert np.array_equal(out[n][2][:small], out[small][2])
    assert np.array_equal(out[huge][1][:big].view(np.uint64), out[big][1].view(np.uint64))


def test_replay_rows_match_the_oracle():
    import torch
    w = netgen.epidemic()
    blob = _blob(w)
    q = api.variable_query(w.var_id, 100, threshold=49, is_max=True)
    params = _random_proposal(8).pack()
    runs = np.array([0, 3, 5, 11, 40], dtype=np.uint64)
    weights = np.array([0.1, 0.2, 0.3, 0.15, 0.25], dtype=np.float32)
    cpu_rows = oracle.is_trace(blob, q, params, 21, runs, weights, first_run=7)
    cpu_out, _ = oracle.is_run(blob, q, params, 21, 41, 7)
    st = cpu_out["steps"][runs.astype(np.int64)].astype(np.int64)
    offs = np.concatenate([[0], np.cumsum(4 * st)[:-1]]).astype(np.uint64)
    assert len(cpu_rows) == int(4 * st.sum())
    net = api.Network(blob)
    P.set_inference(net, False)
    try:
        dev = torch.device("cuda")
        rows = torch.zeros(len(cpu_rows) * P.ROW_BYTES, dtype=torch.uint8, device=dev)
        P.is_trace(net, q, params, 21, torch.from_numpy(runs.view(np.int64)).to(dev),
                   torch.from_numpy(weights).to(dev), torch.from_numpy(offs.view(np.int64)).to(dev), rows, 7)
        got = rows.cpu().numpy().view(oracle.ROW_DTYPE)
    finally:
        net.close()
    assert got.tobytes() == cpu_rows.tobytes()


def _merge_rows_reference(rows, offs):
    """csmc_mlp_rows_merge restated: per run and class, consecutive rows of
    equal features summed (FP64, step order, rounded to FP32); all-zero
    groups dropped; run-major, then class, then first step."""
    out = []
    n = len(rows)
    for i, b in enumerate(offs):
        e = offs[i + 1] if i + 1 < len(offs) else n
        for l in range(4):
            key, head, sa, sb = None, None, 0.0, 0.0
            for r in range(b + l, e, 4):
                x = rows["x"][r].tobytes()
                if x != key:
                    if key is not None and (sa != 0.0 or sb != 0.0):
                        out.append((rows["x"][head], np.float32(sa), np.float32(sb)))
                    key, head, sa, sb = x, r, 0.0, 0.0
                sa += float(rows["a"][r])
                sb += float(rows["b"][r])
            if key is not None and (sa != 0.0 or sb != 0.0):
                out.append((rows["x"][head], np.float32(sa), np.float32(sb)))
    res = np.zeros(len(out), dtype=rows.dtype)
    for k, (x, sa, sb) in enumerate(out):
        res["x"][k] = x
        res["a"][k] = sa
        res["b"][k] = sb
    return res


def test_row_merge_keeps_the_objective_and_gradient():
    """Replayed rows merged on the GPU equal the restated merge byte for byte
    and give the same J and gradient up to rounding."""
    import torch
    w = netgen.epidemic()
    blob = _blob(w)
    q = api.variable_query(w.var_id, 100, threshold=49, is_max=True)
    params = _random_proposal(8).pack()
    runs = np.array([0, 3, 5, 11, 40, 77], dtype=np.uint64)
    weights = np.array([0.1, 0.2, 0.3, 0.15, 0.25, 0.05], dtype=np.float32)
    cpu_rows = oracle.is_trace(blob, q, params, 21, runs, weights, first_run=7)
    cpu_out, _ = oracle.is_run(blob, q, params, 21, 78, 7)
    st = cpu_out["steps"][runs.astype(np.int64)].astype(np.int64)
    offs = np.concatenate([[0], np.cumsum(4 * st)[:-1]]).astype(np.uint64)
    dev = torch.device("cuda")
    rows = torch.from_numpy(cpu_rows.view(np.uint8).copy()).to(dev)
    merged = torch.zeros_like(rows)
    n = P.merge_rows(rows, torch.from_numpy(offs.view(np.int64)).to(dev), len(runs), len(cpu_rows), merged)
    ref = _merge_rows_reference(cpu_rows, [int(o) for o in offs])
    assert n == len(ref) and n < len(cpu_rows) // 2
    got = merged.cpu().numpy()[: n * P.ROW_BYTES].view(oracle.ROW_DTYPE)
    assert got.tobytes() == ref.tobytes()
    g0, j0 = P.mlp_grad(params, rows, len(cpu_rows))
    g1, j1 = P.mlp_grad(params, merged, n)
    assert j1 == pytest.approx(j0, rel=1e-5)
    assert np.linalg.norm(g1 - g0) <= 1e-3 * np.linalg.norm(g0)


def test_row_merge_across_batch_boundaries():
    """Synthetic rows: per chain, features that keep their value from one
    step to the next with probability 0.9 (groups longer than the merge's
    32-step batches, and groups that straddle them), chains of 0 to 200
    steps, a and b zero, negative zero or positive; the GPU merge equals
    the restated merge byte for byte."""
    import torch
    rng = np.random.default_rng(5)
    lens = [0, 1, 31, 32, 33, 64, 65, 200, 7, 0, 96, 150, 0]
    offs = np.concatenate([[0], np.cumsum(4 * np.array(lens))[:-1]]).astype(np.uint64)
    n = 4 * sum(lens)
    rows = np.zeros(n, dtype=oracle.ROW_DTYPE)
    feats = rng.integers(0, 2**16, (3, 16)).astype(np.uint16)
    for b, steps in zip(offs.astype(np.int64), lens):
        for l in range(4):
            cur = int(rng.integers(0, 3))
            for k in range(steps):
                if rng.uniform() > 0.9:
                    cur = int(rng.integers(0, 3))
                rows["x"][b + 4 * k + l] = feats[cur]
    kind = rng.integers(0, 4, (n, 2))
    vals = rng.exponential(1.0, (n, 2)).astype(np.float32)
    ab = np.where(kind == 0, np.float32(-0.0), np.where(kind == 1, np.float32(0.0), vals))
    rows["a"], rows["b"] = ab[:, 0], ab[:, 1]
    dev = torch.device("cuda")
    t_rows = torch.from_numpy(rows.view(np.uint8).copy()).to(dev)
    merged = torch.zeros_like(t_rows)
    got_n = P.merge_rows(t_rows, torch.from_numpy(offs.view(np.int64)).to(dev), len(lens), n, merged)
    ref = _merge_rows_reference(rows, [int(o) for o in offs])
    assert got_n == len(ref)
    assert merged.cpu().numpy()[: got_n * P.ROW_BYTES].tobytes() == ref.tobytes()


def test_tensor_core_inference_follows_the_exact_paths():
    import torch
    w = netgen.epidemic()
    blob = _blob(w)
    q = api.variable_query(w.var_id, 100, threshold=49, is_max=True)
    params = _random_proposal(6).pack()
    n = 4096
    dev = torch.device("cuda")
    out = {}
    net = api.Network(blob)
    try:
        for tc in (False, True):
            P.set_inference(net, tc)
            flags = torch.zeros(n, dtype=torch.uint8, device=dev)
            logw = torch.zeros(n, dtype=torch.float64, device=dev)
            steps = torch.zeros(n, dtype=torch.int32, device=dev)
            P.is_run(net, q, params, 23, n, 0, flags=flags, logw=logw, steps=steps)
            out[tc] = (flags.cpu().numpy(), logw.cpu().numpy(), steps.cpu().numpy())
        # replay under tensor cores reproduces the tensor-core runs
        runs = np.arange(0, 64, dtype=np.uint64)
        st = out[True][2][:64].astype(np.int64)
        offs = np.concatenate([[0], np.cumsum(4 * st)[:-1]]).astype(np.uint64)
        rows = torch.zeros(int(4 * st.sum()) * P.ROW_BYTES, dtype=torch.uint8, device=dev)
        P.is_trace(net, q, params, 23, torch.from_numpy(runs.view(np.int64)).to(dev),
                   torch.ones(64, dtype=torch.float32, device=dev), torch.from_numpy(offs.view(np.int64)).to(dev),
                   rows, 0)
        got = rows.cpu().numpy().view(oracle.ROW_DTYPE)
    finally:
        net.close()
    same = (out[False][2] == out[True][2]) & (out[False][0] == out[True][0])
    assert same.mean() > 0.9, same.mean()
    lw0, lw1 = out[False][1][same], out[True][1][same]
    assert np.max(np.abs(lw0 - lw1)) < 1e-2 * max(1.0, np.max(np.abs(lw0)))
    # every replayed step wrote its four rows (features are never all zero)
    assert np.all(got["x"].any(axis=1))


def _rows(n_runs=64):
    w = netgen.epidemic()
    blob = _blob(w)
    q = api.variable_query(w.var_id, 100, threshold=49, is_max=True)
    prop = _random_proposal(4)
    rng = np.random.default_rng(2)
    rows = oracle.is_trace(blob, q, prop.pack(), 31, np.arange(n_runs), rng.uniform(0.2, 1.0, n_runs))
    return prop, rows


def test_tensor_core_forward_matches_the_oracle():
    import torch
    prop, rows = _rows(16)
    params = prop.pack()
    n = len(rows)
    d_rows = torch.from_numpy(rows.view(np.uint8).copy()).to("cuda")
    theta = torch.zeros(n, dtype=torch.float32, device="cuda")
    P.mlp_forward(params, d_rows, n, theta)
    got = theta.cpu().numpy()
    x = P.bf16_bits_to_f32(rows["x"])
    sample = np.linspace(0, n - 1, 400).astype(int)
    ref = np.array([oracle.mlp_theta(params, x[i]) for i in sample], dtype=np.float32)
    assert np.max(np.abs(got[sample] - ref)) < 1e-2
    assert np.std(ref) > 1e-3  # the rows exercise the network


def test_tensor_core_gradient_matches_the_oracle():
    import torch
    prop, rows = _rows(64)
    params = prop.pack()
    d_rows = torch.from_numpy(rows.view(np.uint8).copy()).to("cuda")
    g_gpu, J_gpu = P.mlp_grad(params, d_rows, len(rows))
    g_cpu, J_cpu = oracle.mlp_grad(params, rows)
    assert J_gpu == pytest.approx(J_cpu, rel=1e-3)
    o = 0
    for name, size in [("w1", 64 * 16), ("b1", 64), ("w2", 64 * 64), ("b2", 64), ("w3", 64), ("b3", 1)]:
        a, b = g_gpu[o:o + size].astype(np.float64), g_cpu[o:o + size].astype(np.float64)
        o += size
        if name == "w1":  # the four one-hot inputs and the six used features; columns 10..15 are zero inputs
            a, b = a.reshape(64, 16)[:, :10].ravel(), b.reshape(64, 16)[:, :10].ravel()
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 2e-2, (name, err)


def test_ce_training_lowers_the_error_of_a_rare_event_estimate():
    w = netgen.epidemic()
    blob = _blob(w)
    # R reaches 90 within T = 80: probability about 5e-4 under the nominal model
    q = api.variable_query(w.var_id, 80, threshold=89, is_max=True)
    net = api.Network(blob)
    try:
        n = 200_000
        p_plain, h_plain, _ = P.estimate(net, q, None, 5, 4_000_000, first_run=900_000_000)
        prop, log = P.train(net, q, seed=1, rounds=6, runs_per_round=50_000, adam_steps=20, lr=5e-3)
        p_is, h_is, _ = P.estimate(net, q, prop, 9, n, first_run=500_000_000)
        p_is0, h_is0, _ = P.estimate(net, q, P.Proposal.init(0), 9, n, first_run=500_000_000)
    finally:
        net.close()
    assert p_plain > 0
    # the untrained proposal is plain SMC; the trained one is much tighter at equal runs
    assert h_is < 0.5 * h_is0 if h_is0 > 0 else h_is < p_is
    assert abs(p_is - p_plain) < 1.5 * (h_is + h_plain), (p_is, h_is, p_plain, h_plain)


def test_c_abi_training_equals_the_python_training():
    """csmc_is_train (the CE loop in the library, for hosts without Python)
    and proposal.train (the loop in Python, its own BF16 packing of the
    runs' parameters) end with the same parameters bit for bit from the same
    initial parameters, and log the same rounds.  Both use the library's
    elite selection (csmc_ce_select), Adam steps (csmc_mlp_adam) and
    kernels."""
    w = netgen.epidemic()
    net = api.Network(_blob(w))
    try:
        q = api.variable_query(w.var_id, 75, threshold=94, is_max=True)
        cfg = dict(rounds=3, runs_per_round=3000, adam_steps=6, lr=3e-2, max_rows=300_000, settle=0)
        prop_py, log_py = P.train(net, q, seed=4, init_seed=0, **cfg)
        prop_c, log_c = P.train_c(net, q, seed=4, init=P.Proposal.init(0), **cfg)
    finally:
        net.close()
    assert np.array_equal(prop_py.vector().view(np.uint32), prop_c.vector().view(np.uint32))
    assert len(log_py.rounds) == len(log_c) == 3
    for a, b in zip(log_py.rounds, log_c):
        assert a["elite"] == b["elite"] and a["rows"] == b["rows"] and a["level"] == b["level"]
        assert a["J_start"] == b["j_start"] and a["J_end"] == b["j_end"] and a["hits"] == b["hits"]
    assert prop_c.pack() == P.Proposal.from_vector(prop_c.vector()).pack()



def _host_adam(x, g, m, v, t, lr):
    """Adam's ascent step in numpy double (csmc_mlp_adam's formulas)."""
    t += 1
    g = np.asarray(g, np.float64)
    m = 0.9 * m + (1 - 0.9) * g
    v = 0.999 * v + (1 - 0.999) * g * g
    mh = m / (1 - 0.9 ** t)
    vh = v / (1 - 0.999 ** t)
    return (x + lr * mh / (np.sqrt(vh) + 1e-8)).astype(np.float32), m, v, t


def test_device_adam_equals_the_host_steps():
    """csmc_mlp_adam (a round's Adam steps on the device, one
    synchronisation) against the same steps on the host: csmc_mlp_grad at
    the host-packed parameters, then Adam's update in numpy double.  The
    master vector, both moments, the step count and the first and last
    objectives of each call are equal bit for bit over two calls (the
    moments carry from one call to the next)."""
    import torch
    n = 50_000
    rng = np.random.default_rng(11)
    x = np.zeros((n, P.IN), np.float32)
    x[np.arange(n), rng.integers(0, 4, n)] = 1.0
    x[:, 5:9] = rng.dirichlet([4, 1, 1, 4], n).astype(np.float32)
    x[:, 9] = rng.uniform(0, 1, n)
    rows = np.zeros(n, dtype=np.dtype([("x", "<u2", (P.IN,)), ("a", "<f4"), ("b", "<f4")]))
    rows["x"] = P.f32_to_bf16_bits(x.ravel()).reshape(n, P.IN)
    rows["a"] = rng.exponential(1e-3, n).astype(np.float32)
    rows["b"] = (rng.uniform(0, 1, n) < 0.3).astype(np.float32) * rng.uniform(0.5, 2.0, n).astype(np.float32)
    dev_rows = torch.from_numpy(rows.view(np.uint8).copy()).cuda()
    lr = 3e-2
    x0 = P.Proposal.init(3).vector()
    xd = x0.copy()
    state = P.AdamState()
    ja = P.adam_run(dev_rows, n, 5, lr, xd, state)
    jb = P.adam_run(dev_rows, n, 3, lr, xd, state)
    xh, m, v, t = x0.copy(), np.zeros(P.GRAD_FLOATS), np.zeros(P.GRAD_FLOATS), 0
    Js = []
    for _ in range(8):
        g, J = P.mlp_grad(P.Proposal.from_vector(xh).pack(), dev_rows, n)
        Js.append(J)
        xh, m, v, t = _host_adam(xh, g, m, v, t, lr)
    assert state.t == t == 8
    assert np.array_equal(xd.view(np.uint32), xh.view(np.uint32))
    assert np.array_equal(state.m.view(np.uint64), m.view(np.uint64))
    assert np.array_equal(state.v.view(np.uint64), v.view(np.uint64))
    assert ja == (Js[0], Js[4]) and jb == (Js[5], Js[7])
    assert not np.array_equal(x0, xh)


@pytest.mark.parametrize("case", ["epidemic_permuted", "mutex_clock"])
def test_feature_source_is_a_network_choice(case):
    """A non-default feature source (csmc_is_set_features): the epidemic's
    counts in another order and scale, and a mutex network whose features
    are its shared variables and one process's clock.  Runs and replay rows
    stay bit-identical to the oracle given the same source."""
    import torch
    if case == "epidemic_permuted":
        w, T, thr = netgen.epidemic(), 100, 49
        src = dict(count_vars=[3, 2, 1, 0], scales=[0.02, 0.5 / 100, 0.01, 0.03], clock_var=-1)
    else:
        w, T, thr = netgen.mutex(8), None, None
        src = dict(count_vars=[1, 0, -1, -1], scales=[0.5, 0.125, 1.0, 1.0], clock_var=2)
    blob = _blob(w)
    info = api.blob_info(blob)
    q = api.variable_query(w.var_id, T or w.horizon, threshold=thr if thr is not None else w.threshold,
                           is_max=True, max_steps=100_000)
    params = _random_proposal(5).pack()
    feats = P.pack_features(info["n_vars"], info["n_comps"], **src)
    n = 384
    net = api.Network(blob)
    P.set_inference(net, False)
    P.set_features(net, **src)
    try:
        dev = torch.device("cuda")
        flags = torch.zeros(n, dtype=torch.uint8, device=dev)
        logw = torch.zeros(n, dtype=torch.float64, device=dev)
        steps = torch.zeros(n, dtype=torch.int32, device=dev)
        P.is_run(net, q, params, 23, n, 7, flags=flags, logw=logw, steps=steps)
        cpu, _ = oracle.is_run(blob, q, params, 23, n, 7, features=feats)
        assert np.array_equal(flags.cpu().numpy(), cpu["flags"])
        assert np.array_equal(steps.cpu().numpy().view(np.uint32), cpu["steps"])
        assert np.array_equal(logw.cpu().numpy().view(np.uint64), cpu["logw"].view(np.uint64))
        # the default source gives other paths once theta differs (sanity)
        cpu_default, _ = oracle.is_run(blob, q, params, 23, n, 7)
        assert not np.array_equal(cpu_default["logw"], cpu["logw"])
        # replay rows of a few runs
        runs = np.arange(0, 16, dtype=np.uint64)
        wts = np.full(16, 1.0 / 16, np.float32)
        st = cpu["steps"][:16].astype(np.uint64)
        offs = np.concatenate([[0], np.cumsum(4 * st)[:-1]]).astype(np.uint64)
        n_rows = int(4 * st.sum())
        rows = torch.zeros(n_rows * P.ROW_BYTES, dtype=torch.uint8, device=dev)
        P.is_trace(net, q, params, 23, torch.from_numpy(runs.view(np.int64)).to(dev), torch.from_numpy(wts).to(dev),
                   torch.from_numpy(offs.view(np.int64)).to(dev), rows, 7)
        want = oracle.is_trace(blob, q, params, 23, runs, wts, 7, cap=n_rows, features=feats)
        assert rows.cpu().numpy().tobytes() == want.tobytes()
    finally:
        net.close()
