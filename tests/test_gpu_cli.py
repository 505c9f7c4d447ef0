"""The drop-in CLI on the GPU: the reference's report lines, exit code and
timing CSV (main.cu, smc.cu:283-491, simulation/write_csv.cu), and this
build's extensions: a query given as an UPPAAL formula, the JSON summary and
the per-run CSV, whose numbers must be those of csmc_run for the same seed."""
import csv
import json
import os
import re
import subprocess

import numpy as np
import pytest

from cusmc_b200 import api, netgen

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cusmc_b200", "bin", "cusmc")


def _run(args, cwd):
    return subprocess.run([CLI, *args], cwd=cwd, capture_output=True, text=True, timeout=300)


def test_reference_report_and_timing_csv(tmp_path):
    w = netgen.epidemic(n_agents=30)
    model = w.write(str(tmp_path / "epi.xml"))
    run = tmp_path / "run"
    run.mkdir()
    p = _run(["-m", model, "-s", "7", "-q", "4096", "100", "14", "3", "1", "0", ""], run)
    assert p.returncode == 1, p.stderr
    assert "Set number of variables to: 4" in p.stdout
    assert "- Number of simulations: 4096" in p.stdout
    res = float(re.search(r"^Result: (\S+)", p.stdout, re.M).group(1))
    assert 0.0 < res < 1.0
    assert re.search(r"^Time taken: \S+ ms on file ", p.stdout, re.M)
    # write_csv.cu layout: header row with an empty corner cell, then one
    # column per MC<components>_Sim<runs>_Time<T> configuration; one row per
    # model file with the time in ms
    rows = list(csv.reader(open(tmp_path / "results5.csv"), delimiter=";"))
    assert rows[0][0] == "" and rows[0][1] == "MC30_Sim4096_Time100.00"
    row = next(r for r in rows[1:] if r[0] == "epi.xml")
    assert float(row[1]) > 0.0


def test_formula_json_and_run_dump_match_the_library(tmp_path):
    w = netgen.epidemic(n_agents=30)
    model = w.write(str(tmp_path / "epi.xml"))
    run = tmp_path / "run"
    run.mkdir()
    js, runs = tmp_path / "out.json", tmp_path / "runs.csv"
    p = _run(["-m", model, "-s", "11", "--csmc-formula", "Pr[<=100; 3000](<> R >= 15)", "--csmc-json", str(js),
              "--csmc-runs-csv", str(runs)], run)
    assert p.returncode == 1, p.stderr
    d = json.load(open(js))
    assert d["simulations"] == 3000 and d["query"]["var_id"] == 3 and d["query"]["is_max"] == 1
    lo, hi = d["ci95"]
    assert lo <= d["result"] <= hi and d["chernoff_hoeffding"]["epsilon"] > 0
    table = np.genfromtxt(runs, delimiter=",", names=True)
    assert len(table) == 3000
    # the same runs through the library
    blob = api.compile_model(model)
    q, _, _ = api.parse_query(model, "Pr[<=100](<> R >= 15)")
    r, flags, values, _ = api.run_host(blob, q, 11, 3000)
    assert d["result"] == pytest.approx(r.hits / 3000, abs=0)
    assert np.array_equal(table["value"], values)


def test_importance_sampling_from_the_command_line(tmp_path):
    """--csmc-is: CE training through the C ABI, then weighted runs; the
    estimate agrees with plain SMC on an event that plain SMC sees often."""
    w = netgen.epidemic(n_agents=30)
    model = w.write(str(tmp_path / "epi.xml"))
    run = tmp_path / "run"
    run.mkdir()
    js = tmp_path / "is.json"
    p = _run(["-m", model, "-s", "3", "-q", "20000", "60", "9", "3", "1", "0", "", "--csmc-is",
              "--csmc-is-ce", "3,3000,5,0.03", "--csmc-json", str(js)], run)
    assert p.returncode == 1, p.stderr
    assert "Importance sampling: learned proposal, up to 3 CE rounds of 3000 runs" in p.stdout
    assert re.search(r"^CE round 0: level ", p.stdout, re.M)
    out = json.load(open(js))
    assert out["method"].startswith("importance sampling") and out["simulations"] == 20000
    lo, hi = out["ci95"]
    blob = api.compile_model(model)
    net = api.Network(blob)
    try:
        r = net.run(api.variable_query(3, 60, threshold=9, is_max=True), 77, 400_000)
    finally:
        net.close()
    half_plain = 1.96 * np.sqrt(r.estimate * (1 - r.estimate) / 400_000)
    assert lo - half_plain <= r.estimate <= hi + half_plain
    # an estimate query (IS_ESTIMATE = 1) has no probability to sample: refused with an error
    p = _run(["-m", model, "-q", "1000", "60", "9", "3", "1", "1", "", "--csmc-is"], run)
    assert "Error:" in p.stderr
