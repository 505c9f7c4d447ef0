"""UPPAAL query formulas -> simulation queries (csmc_query_parse), on CPU.

The reference ignores its models' <queries> and takes the query from its
command line; this library reads the SMC subset those formulas use.  The
fixture cases run only where the reference's model files are present."""
import math
import os

import pytest

from cusmc_b200 import api, netgen

# the reference checkout (read-only); CSMC_REFERENCE overrides the default location
REF_XML = os.path.join(os.environ.get("CSMC_REFERENCE", "/root/reference"), "xml_files")


def _q(path, formula):
    return api.parse_query(path, formula)


def test_variable_reachability_and_estimates(tmp_path):
    w = netgen.epidemic(n_agents=10)
    path = w.write(str(tmp_path / "e.xml"))
    q, loc, n = _q(path, "Pr[<=100](<> R >= 5)")
    assert (q.kind, q.var_id, q.is_max, q.is_estimate, q.horizon, loc, n) == (1, 3, 1, 0, 100.0, "", 0)
    assert q.threshold < 5 and math.nextafter(q.threshold, math.inf) == 5.0  # max > t  <=>  max >= 5
    q, _, _ = _q(path, "Pr[<=50; 2000](<> I > 3)")
    assert (q.var_id, q.is_max, q.threshold, q.horizon) == (2, 1, 3.0, 50.0)
    q, _, _ = _q(path, "Pr[<=50](<> S <= 2)")
    assert (q.var_id, q.is_max) == (0, 0) and q.threshold > 2 and math.nextafter(q.threshold, -math.inf) == 2.0
    q, _, n = _q(path, "E[<=100; 5000](min: S)")
    assert (q.kind, q.var_id, q.is_max, q.is_estimate, n) == (1, 0, 0, 1, 5000)


def test_location_reachability_by_template_and_local_variables(tmp_path):
    w = netgen.mutex(4)
    path = w.write(str(tmp_path / "m.xml"))
    q, loc, _ = _q(path, "Pr[<=200](<> P2.cs)")
    assert (q.kind, q.var_id, loc, q.horizon) == (0, -1, "P2.cs", 200.0)
    q, _, _ = _q(path, "Pr[<=200](<> P1.x >= 3)")  # a template-local clock
    assert q.var_id >= 2


@pytest.mark.parametrize("formula,msg", [
    ("A[] not deadlock", "only Pr"),
    ("Pr[<=300](<> P(1).cs)", "parameterised"),
    ("Pr[<=10](<> nope >= 1)", "no variable"),
    ("Pr[<=10](<> P0.nowhere)", "no location"),
    ("E[<=10](max: id)", "run count"),
    ("Pr[<=10](<> id == 1)", "equality"),
    ("Pr[<=nan](<> id >= 1)", "time bound must be a finite number"),
    ("Pr[<=inf](<> id >= 1)", "time bound must be a finite number"),
    ("Pr[<=-5](<> id >= 1)", "must not be negative"),
    ("Pr[<=10](<> id >= nan)", "threshold must be a finite number"),
    ("Pr[<=10; 0](<> id >= 1)", "positive integer"),
    ("Pr[<=10; 2.5](<> id >= 1)", "positive integer"),
    ("Pr[<=10; 99999999999999999999999](<> id >= 1)", "at most 2^53"),
    ("Pr[<=1e400](<> id >= 1)", "not a number"),
])
def test_unsupported_formulas_are_rejected(tmp_path, formula, msg):
    path = netgen.mutex(2).write(str(tmp_path / "m.xml"))
    with pytest.raises(api._native.CsmcError) as e:
        _q(path, formula)
    assert msg in str(e.value)


@pytest.mark.skipif(not os.path.isdir(REF_XML), reason="the reference's model files are not present")
@pytest.mark.parametrize("model,formula,expect", [
    ("LargeModels/aloha_50.xml", "E[<=100; 10240](max: nt)", (1, 1, 1, 100.0, "", 10240)),
    ("LargeModels/fischer_10_29.xml", "E[<=300; 1000](max: in_critical)", (1, 1, 1, 300.0, "", 1000)),
    ("UppaalBehaviorTest3.xml", "Pr[<=100] (<> c1.f2)", (0, 1, 0, 100.0, "c1.f2", 0)),
    ("bluetoothSmacc.xml", "Pr[<=5000; 10240](<> receiver1.Reply)", (0, 1, 0, 5000.0, "Receiver.Reply", 10240)),
])
def test_the_reference_fixture_formulas(model, formula, expect):
    q, loc, n = _q(os.path.join(REF_XML, model), formula)
    assert (q.kind, q.is_max, q.is_estimate, q.horizon, loc, n) == expect
