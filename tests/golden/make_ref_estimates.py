"""Runs the REFERENCE cuSMC binary (oracle/_ref/cusmc_ref_v*, built from the
reference sources for sm_100a by oracle/ref/Makefile) on a fixed list of
models and queries and records its estimates in tests/golden/ref_estimates.json.
Needs a GPU; run from the repository root:

  python tests/golden/make_ref_estimates.py --models <dir with the reference's xml_files> [--out FILE]

Only models that are safe for the reference kernel are listed: none of them
reaches a clock invariant with no enabled edge (the reference kernel would
then propose a zero delay forever, e.g. UppaalBehaviorTest2) and no location
has two receiving edges that can be enabled together (the reference then
draws from an invalid random-state pointer).  Each model runs with the
smallest MAX_VARIABLES build that holds its variables.

The estimates pin the CPU oracle's simulation semantics statistically
(tests/test_ref_estimates.py); the reference's own random streams are not
reproducible run by run (its curand states are shared by all blocks).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cusmc_b200 import api, netgen  # noqa: E402

# (name, model source, -q arguments without the simulation count, sims, seed)
#   -q arguments: T threshold var_id is_max is_estimate loc_query
CASES = [
    ("epidemic_100", "gen:epidemic", ["100", "49", "3", "1", "0", ""], 400_000, 11),
    ("random_0", "gen:random_0", ["100", "12", "0", "1", "0", ""], 1_000_000, 12),
    ("random_2", "gen:random_2", ["100", "10", "0", "1", "0", ""], 1_000_000, 14),
    ("random_3", "gen:random_3", ["100", "12", "0", "1", "0", ""], 1_000_000, 15),
    ("mutex_8", "gen:mutex_8", ["5", "0", "1", "1", "0", ""], 1_000_000, 16),
    ("mutex_32", "gen:mutex_32", ["5", "0", "1", "1", "0", ""], 1_000_000, 17),
    ("agentBaseCovid_100_1.0", "agentBaseCovid_100_1.0.xml", ["100", "20", "1", "1", "0", " "], 100_000, 18),
    ("agentBaseCovid_32_1", "agentBaseCovid_32_1.xml", ["100", "10", "1", "1", "0", ""], 300_000, 19),
    ("aloha_25_loc", "LargeModels/aloha_25.xml", ["1", "-1", "-1", "1", "0", "P0.Transmit"], 1_000_000, 20),
    ("fischer_10_29_loc", "LargeModels/fischer_10_29.xml", ["100", "-1", "-1", "1", "0", "P3.cs"], 300_000, 21),
    ("condTest_loc", "condTest.xml", ["100", "-1", "-1", "1", "0", "Template.l3"], 1_000_000, 22),
    ("UppaalWeightTest_loc", "UppaalWeightTest.xml", ["10", "-1", "-1", "1", "0", "Template.l4"], 1_000_000, 23),
    ("RaceTest_est", "RaceTest.xml", ["100", "0", "0", "1", "1", ""], 100_000, 24),
    ("fischermulti_loc", "fischermulti.xml", ["10", "-1", "-1", "1", "0", "P1.cs"], 1_000_000, 25),
]


def generated(name: str, d: str) -> str:
    w = {"epidemic": lambda: netgen.epidemic(), "mutex_8": lambda: netgen.mutex(8),
         "mutex_32": lambda: netgen.mutex(32)}.get(name)
    if w is None:
        w = lambda: netgen.random_network(int(name.split("_")[1]))  # noqa: E731
    return w().write(os.path.join(d, name + ".xml"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--models", required=True, help="directory of the reference's xml_files")
    ap.add_argument("--out", default=os.path.join(HERE, "ref_estimates.json"))
    args = ap.parse_args()
    tmp = tempfile.mkdtemp(prefix="csmc_refest_")
    cwd = os.path.join(tmp, "run")  # the reference writes ../results5.csv
    os.makedirs(cwd)
    out = {"command": "python tests/golden/make_ref_estimates.py --models <reference xml_files>", "cases": []}
    for name, src, qargs, sims, seed in CASES:
        path = generated(src[4:], tmp) if src.startswith("gen:") else os.path.join(os.path.abspath(args.models), src)
        loc_mode = qargs[2] == "-1"  # var_id == -1
        info = api.blob_info(api.compile_model(path, qargs[5], loc_mode))
        variant = next(v for v in (8, 16, 64, 512) if v >= info["n_vars"])
        binary = os.path.join(ROOT, "oracle", "_ref", f"cusmc_ref_v{variant}")
        cmd = [binary, "-m", path, "-s", str(seed), "-q", str(sims)] + qargs
        t0 = time.time()
        p = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=900)
        dt = time.time() - t0
        text = p.stdout
        entry = {"name": name, "model": src, "query": qargs, "sims": sims, "seed": seed,
                 "binary": os.path.basename(binary), "wall_s": round(dt, 2), "exit": p.returncode}
        m = re.search(r"^Result: (\S+)", text, re.M)
        if m:
            entry["result"] = float(m.group(1))
        m = re.search(r"^Number of hits: (\d+)", text, re.M)
        if m:
            entry["hits"] = int(m.group(1))
            entry["result"] = int(m.group(1)) / sims
        m = re.search(r"^Time taken: ([0-9.e+-]+) ms on file", text, re.M)
        if m:
            entry["kernel_ms"] = float(m.group(1))
        if "result" not in entry:
            entry["tail"] = (text + p.stderr)[-400:]
        out["cases"].append(entry)
        print(json.dumps(entry), flush=True)
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
