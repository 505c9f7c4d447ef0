"""The front end behind the C ABI on malformed input: seeded mutations of
generated models (truncations, spliced tokens, deleted and replaced spans)
either compile or come back as CSMC_ERR_MODEL with a message; nothing
crashes the process, and every mutant that compiles runs in the CPU oracle.
The loop runs in a child process so that a crash shows up as a failed test
rather than as a dead test session."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import ctypes, json, os, random, sys, tempfile
sys.path.insert(0, sys.argv[1])
import oracle
from cusmc_b200 import _native, api, netgen
lib = _native.lib()
rng = random.Random(int(sys.argv[2]))
bases = [netgen.epidemic(n_agents=5).xml, netgen.mutex(4).xml, netgen.random_network(3).xml]
tokens = ['<', '>', '&amp;', '&lt;', '"', "'", '(', ')', '+', '-', '*', '/', '%', '==', '!=', '<=', '>=',
          '&&', '||', '!', '?', ':', ',', ';', '=', ':=', '[', ']', '{', '}', 'x', '0', '1', '1e308', '-1e308',
          'nan', '999999999999', 'const', 'int', 'clock', 'double', 'chan', 'broadcast', 'sqrt', 'pow',
          'random', ' ', '\n', '</', '/>', '<location', '<transition', '<label', 'kind="guard"']
codes, ran = {}, 0
path = os.path.join(tempfile.mkdtemp(), 'm.xml')
for i in range(int(sys.argv[3])):
    s = rng.choice(bases)
    k = rng.randrange(4)
    if k == 0:
        s = s[:rng.randrange(len(s) + 1)]
    elif k == 1:
        for _ in range(rng.randrange(1, 6)):
            p = rng.randrange(len(s) + 1)
            s = s[:p] + rng.choice(tokens) + s[p:]
    elif k == 2:
        for _ in range(rng.randrange(1, 4)):
            p = rng.randrange(len(s) + 1)
            s = s[:p] + s[min(len(s), p + rng.randrange(40)):]
    else:
        for _ in range(rng.randrange(1, 4)):
            p = rng.randrange(len(s) + 1)
            s = s[:p] + ''.join(rng.choice(tokens) for _ in range(rng.randrange(1, 5))) + s[p + rng.randrange(10):]
    with open(path, 'w') as f:
        f.write(s)
    blob = ctypes.c_void_p()
    nb = ctypes.c_size_t()
    rc = lib.csmc_model_compile(path.encode(), b'', 0, ctypes.byref(blob), ctypes.byref(nb))
    codes[str(rc)] = codes.get(str(rc), 0) + 1
    if rc != 0:
        assert rc == _native.CSMC_ERR_MODEL, rc
        assert lib.csmc_last_error(), 'an error without a message'
        continue
    data = ctypes.string_at(blob, nb.value)
    lib.csmc_free(blob)
    if api.blob_info(data)['n_vars'] > 0:
        oracle.run(data, api.variable_query(0, 20, threshold=3, is_max=True, max_steps=2000), 7, 2, threads=1)
        ran += 1
print(json.dumps({'codes': codes, 'ran': ran}))
'''


def _fuzz(seed, n):
    p = subprocess.run([sys.executable, '-c', CHILD, ROOT, str(seed), str(n)], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert p.returncode == 0, (p.returncode, p.stderr[-2000:])
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_mutated_models_compile_or_fail_cleanly():
    out = _fuzz(5, 600)
    assert sum(out['codes'].values()) == 600
    assert out['codes'].get('0', 0) > 0 and out['codes'].get(str(-2), 0) > 0  # both outcomes exercised
    assert out['ran'] > 0


def test_mutated_formulas_parse_or_fail_cleanly(tmp_path):
    import random

    from cusmc_b200 import _native, api, netgen
    path = netgen.epidemic(n_agents=5).write(str(tmp_path / "e.xml"))
    good = ["Pr[<=100](<> R >= 3)", "Pr[<=50; 1000](<> Agent1.I)", "E[<=80; 500](max: R)", "Pr[<=10](<> S < 2)"]
    pieces = ["[", "]", "(", ")", "<=", ">=", "<", ">", "==", "!=", ";", ",", ":", "<>", "[]", "max", "min", "Pr",
              "E", "R", "S", "Agent1", ".", "I", "-1", "1e400", "nan", "99999999999999999999", " ", "\t", "x", "#"]
    rng = random.Random(3)
    outcomes = {"ok": 0, "err": 0}
    for _ in range(2000):
        f = rng.choice(good)
        for _ in range(rng.randrange(1, 4)):
            p = rng.randrange(len(f) + 1)
            f = f[:p] + rng.choice(pieces) + f[p + rng.randrange(4):]
        try:
            q, loc, sims = api.parse_query(path, f)
        except _native.CsmcError as e:
            assert e.code in (_native.CSMC_ERR_ARG, _native.CSMC_ERR_MODEL), (f, e.code)
            outcomes["err"] += 1
            continue
        assert q.kind in (_native.QUERY_LOCATION, _native.QUERY_VARIABLE)
        assert q.kind == _native.QUERY_LOCATION or 0 <= q.var_id < api.blob_info(api.compile_model(path))["n_vars"]
        outcomes["ok"] += 1
    assert outcomes["ok"] > 0 and outcomes["err"] > 0, outcomes
