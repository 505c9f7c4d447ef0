"""Regenerates the golden fixtures under tests/golden/ (run from the repo root
in the build container, where the reference checkout and its build exist):

  python tests/golden/make_golden.py [--ref REFERENCE_CHECKOUT]   (default: $CSMC_REFERENCE)

* frontend/<model>.<mode>.dump — the network as the REFERENCE front end
  delivers it to its kernel (oracle/_ref/refdump: reference parser, optimizer,
  PN compiler and variable registry; location-query goal marking for "loc"),
  in the canonical dump format.  tests/test_frontend.py checks this library's
  front end against them.
* nets/<model>.<mode>.blob — this library's packed network for the same model
  and query, so GPU parity tests can run the reference's model files on a box
  without the reference checkout.
* manifest.json — the models, queries and the command that produced each file.

Generated networks are not stored: tests regenerate them from their seeds
with cusmc_b200.netgen (the generators are deterministic).

Models: every file of the reference's xml_files/ and xml_files/LargeModels/
plus the seeded benchmark networks of cusmc_b200.netgen.
"""
from __future__ import annotations

import argparse
import gzip
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cusmc_b200 import api, netgen  # noqa: E402

# (model relative to xml_files/, location query used for the "loc" dump)
FIXTURES = [
    ("RaceTest.xml", "Template7.id1"),
    ("UppaalBehaviorTest2.xml", "c1.f2"),
    ("UppaalBehaviorTest3.xml", "c1.f2"),
    ("UppaalWeightTest.xml", "Template.l4"),
    ("agentBaseCovid_32_1.xml", "person0.S"),
    ("agentBaseCovid_100_1.0.xml", " "),
    ("agentBaseCovid_350.xml", ""),
    ("bluetoothSmacc.xml", ""),
    ("condTest.xml", "Process.l3"),
    ("fischermulti.xml", "P1.cs"),
    ("LargeModels/CSMA_100.xml", ""),
    ("LargeModels/aloha_25.xml", "P0.Transmit"),
    ("LargeModels/aloha_50.xml", "P3.Transmit"),
    ("LargeModels/fischer_10_29.xml", "P3.cs"),
    ("LargeModels/fischer_100_29.xml", "P0.cs"),
]


# expression-zoo seeds whose models the reference front end accepts (the
# reference-subset generator and the full one)
ZOO_SEEDS = [0, 1, 2, 4, 5]
ZOO_FULL_SEEDS = [60, 73]


def generated():
    ws = [netgen.epidemic(), netgen.mutex(8), netgen.mutex(32)]
    ws += [netgen.random_network(s) for s in range(4)]
    ws += netgen.batch_networks(6)
    ws += [netgen.expression_zoo(s) for s in ZOO_SEEDS]
    ws += [netgen.expression_zoo(s, full=True) for s in ZOO_FULL_SEEDS]
    return ws


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("CSMC_REFERENCE", "/root/reference"))
    args = ap.parse_args()
    refdump = os.path.join(ROOT, "oracle", "_ref", "refdump")
    if not os.path.exists(refdump):
        sys.exit("build oracle/_ref/refdump first: make -f oracle/ref/Makefile REF=" + args.ref)
    os.makedirs(os.path.join(HERE, "frontend"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "nets"), exist_ok=True)
    gen_dir = tempfile.mkdtemp(prefix="csmc_gen_")
    manifest = {"command": "python tests/golden/make_golden.py --ref " + args.ref, "models": []}
    items = [(os.path.join(args.ref, "xml_files", rel), os.path.basename(rel)[:-4], lq) for rel, lq in FIXTURES]
    for w in generated():
        path = w.write(os.path.join(gen_dir, w.name + ".xml"))
        items.append((path, w.name, ""))
    for path, name, lq in items:
        for mode, query in (("var", lq), ("loc", lq)):
            out = subprocess.run([refdump, path, query, mode], capture_output=True, text=True)
            dump = out.stdout
            with open(os.path.join(HERE, "frontend", f"{name}.{mode}.dump.gz"), "wb") as raw:
                with gzip.GzipFile(fileobj=raw, mode="wb", mtime=0) as f:  # reproducible bytes
                    f.write(dump.encode())
            entry = {"name": name, "mode": mode, "loc_query": query, "ref_status": out.returncode,
                     "generated": path.startswith(gen_dir)}
            if out.returncode == 0:
                blob = api.compile_model(path, query, mode == "loc")
                entry.update(api.blob_info(blob))
                if not entry["generated"]:
                    with open(os.path.join(HERE, "nets", f"{name}.{mode}.blob"), "wb") as f:
                        f.write(blob)
            manifest["models"].append(entry)
            print(name, mode, out.returncode, len(dump))
    # packed networks of the reference-estimate cases (make_ref_estimates.py),
    # compiled with exactly the query each reference run used
    import importlib.util
    spec = importlib.util.spec_from_file_location("refest", os.path.join(HERE, "make_ref_estimates.py"))
    refest = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(refest)
    for name, src, qargs, _sims, _seed in refest.CASES:
        if src.startswith("gen:"):
            continue
        path = os.path.join(args.ref, "xml_files", src)
        blob = api.compile_model(path, qargs[5], qargs[2] == "-1")
        with open(os.path.join(HERE, "nets", f"refest_{name}.blob"), "wb") as f:
            f.write(blob)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
