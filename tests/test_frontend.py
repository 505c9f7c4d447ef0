"""Front-end parity: this library's front end against the REFERENCE front end
(parser, optimizer, PN compiler, variable registry, location-query goal
marking), compared on the canonical dump of the network each delivers to its
kernel.  The reference side is committed under tests/golden/frontend (made by
tests/golden/make_golden.py from oracle/_ref/refdump).
"""
import gzip
import json
import os
import tempfile

import pytest

from conftest import GOLDEN
from cusmc_b200 import api, netgen

# the reference checkout (read-only); CSMC_REFERENCE overrides the default location
REF_XML = os.path.join(os.environ.get("CSMC_REFERENCE", "/root/reference"), "xml_files")

with open(os.path.join(GOLDEN, "manifest.json")) as f:
    MANIFEST = json.load(f)


def _golden(name, mode):
    with gzip.open(os.path.join(GOLDEN, "frontend", f"{name}.{mode}.dump.gz"), "rt") as f:
        return f.read()


def _generated():
    ws = {w.name: w for w in [netgen.epidemic(), netgen.mutex(8), netgen.mutex(32)]}
    ws.update({w.name: w for w in [netgen.random_network(s) for s in range(4)]})
    ws.update({w.name: w for w in netgen.batch_networks(6)})
    for m in MANIFEST["models"]:  # expression-zoo models: zoo_<seed>, zoo_full_<seed>
        if m["generated"] and m["name"].startswith("zoo_"):
            full = m["name"].startswith("zoo_full_")
            w = netgen.expression_zoo(int(m["name"].rsplit("_", 1)[1]), full=full)
            ws[w.name] = w
    return ws


GENERATED = _generated()


@pytest.mark.parametrize("entry", [m for m in MANIFEST["models"] if m["generated"]],
                         ids=lambda m: f"{m['name']}-{m['mode']}")
def test_generated_models_match_reference_front_end(entry):
    w = GENERATED[entry["name"]]
    with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
        f.write(w.xml)
        path = f.name
    try:
        got = api.dump_model(path, entry["loc_query"], entry["mode"] == "loc")
    finally:
        os.unlink(path)
    assert got == _golden(entry["name"], entry["mode"])


@pytest.mark.skipif(not os.path.isdir(REF_XML), reason="reference model files not present")
@pytest.mark.parametrize("entry", [m for m in MANIFEST["models"] if not m["generated"]],
                         ids=lambda m: f"{m['name']}-{m['mode']}")
def test_reference_fixtures_match_reference_front_end(entry):
    name = entry["name"]
    rel = name + ".xml"
    path = os.path.join(REF_XML, rel)
    if not os.path.exists(path):
        path = os.path.join(REF_XML, "LargeModels", rel)
    got = api.dump_model(path, entry["loc_query"], entry["mode"] == "loc")
    assert got == _golden(name, entry["mode"])
    blob = api.compile_model(path, entry["loc_query"], entry["mode"] == "loc")
    with open(os.path.join(GOLDEN, "nets", f"{name}.{entry['mode']}.blob"), "rb") as f:
        assert blob == f.read()


def test_unreachable_location_is_rejected_like_the_reference():
    # the reference's upload throws std::out_of_range for a location that the
    # optimizer never visited (shared_model_state.cu:475)
    xml = netgen.epidemic(n_agents=3).xml.replace('<init ref="id0"/>', '<init ref="id1"/>', 1)
    with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
        f.write(xml)
        path = f.name
    try:
        with pytest.raises(api._native.CsmcError):
            api.compile_model(path)
    finally:
        os.unlink(path)


def test_missing_file_is_a_model_error():
    with pytest.raises(api._native.CsmcError) as e:
        api.compile_model("/nonexistent/model.xml")
    assert e.value.code == api._native.CSMC_ERR_MODEL


REFDUMP = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "refdump")


@pytest.mark.skipif(not os.path.exists(REFDUMP), reason="the reference front-end dump tool is not built")
@pytest.mark.parametrize("full", [False, True], ids=["reference-subset", "full"])
def test_expression_zoo_matches_reference_front_end(tmp_path, full):
    """Differential check against the reference's own parser, optimizer and
    PN compiler (oracle/_ref/refdump) on 60 random expression-zoo models:
    both accept with byte-identical networks, or both reject."""
    import subprocess
    from cusmc_b200 import _native
    outcome = {"match": 0, "both_reject": 0}
    for seed in range(60, 120) if full else range(60):
        w = netgen.expression_zoo(seed, full=full)
        path = w.write(str(tmp_path / f"{w.name}.xml"))
        ref = subprocess.run([REFDUMP, path, "", "var"], capture_output=True, text=True, timeout=120)
        try:
            ours = api.dump_model(path, "", False)
        except _native.CsmcError:
            ours = None
        if ref.returncode == 0:
            assert ours is not None, f"seed {seed}: the reference accepts, this front end rejects"
            assert ours == ref.stdout, f"seed {seed}: the networks differ"
            outcome["match"] += 1
        else:
            assert ours is None, f"seed {seed}: the reference rejects, this front end accepts"
            outcome["both_reject"] += 1
    assert outcome["match"] > 0 and outcome["both_reject"] > 0, outcome
