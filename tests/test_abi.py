"""The C ABI boundary without a GPU: libcsmc.so loads, exports every entry
point include/csmc.h declares, the ctypes table binds exactly those, the
calls that need no device work on the host, and the CLI keeps the
reference's argument handling and exit codes (main.cu:10-110: 0 after -h or
an argument error, 1 after a simulation attempt)."""
import ctypes
import os
import re
import subprocess

import pytest

from cusmc_b200 import _native, api, netgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "csmc.h")
CLI = os.path.join(ROOT, "cusmc_b200", "bin", "cusmc")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(csmc_[a-z_]+)\s*\(", text)))


def test_every_declared_entry_point_is_exported_and_bound():
    names = _declared()
    assert len(names) >= 20
    lib = _native.lib()
    for name in names:
        assert hasattr(lib, name), f"{name} is declared but not exported"
    assert sorted(_native.exported_symbols()) == names


def test_host_side_calls_work_without_a_device(tmp_path):
    w = netgen.mutex(8)
    path = w.write(str(tmp_path / "m.xml"))
    blob = api.compile_model(path)
    info = api.blob_info(blob)
    assert info["n_comps"] == 8
    assert api.version().startswith("csmc-b200")


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-device error path")
def test_upload_without_a_device_fails_loudly(tmp_path):
    w = netgen.mutex(8)
    blob = api.compile_model(w.write(str(tmp_path / "m.xml")))
    with pytest.raises(_native.CsmcError) as e:
        api.Network(blob)
    assert e.value.code == _native.CSMC_ERR_NODEVICE


def test_adam_entry_point_checks_its_arguments_first():
    """csmc_mlp_adam refuses a missing master vector or moment array and a
    step count below one before it touches a device."""
    import numpy as np
    from cusmc_b200 import proposal as P
    lib = _native.lib()
    x = np.zeros(P.GRAD_FLOATS, np.float32)
    m = np.zeros(P.GRAD_FLOATS, np.float64)
    v = np.zeros(P.GRAD_FLOATS, np.float64)
    t = ctypes.c_int32(0)
    j0, j1 = ctypes.c_double(), ctypes.c_double()
    assert lib.csmc_mlp_adam(None, 0, 0, 1e-2, x.ctypes.data, m.ctypes.data, v.ctypes.data, ctypes.byref(t),
                             ctypes.byref(j0), ctypes.byref(j1), None) == _native.CSMC_ERR_ARG
    assert lib.csmc_mlp_adam(None, 0, 3, 1e-2, None, m.ctypes.data, v.ctypes.data, ctypes.byref(t),
                             ctypes.byref(j0), ctypes.byref(j1), None) == _native.CSMC_ERR_ARG
    assert lib.csmc_mlp_adam(None, 5, 3, 1e-2, x.ctypes.data, m.ctypes.data, v.ctypes.data, ctypes.byref(t),
                             ctypes.byref(j0), ctypes.byref(j1), None) == _native.CSMC_ERR_ARG
    assert t.value == 0


def _cli(*args, cwd=None):
    return subprocess.run([CLI, *args], capture_output=True, text=True, cwd=cwd, timeout=60)


def test_cli_help_exits_zero():
    p = _cli("-h")
    assert p.returncode == 0
    assert "-m or --model" in p.stdout


@pytest.mark.parametrize("args", [["-m"], ["-s", "x"], ["-q", "10", "10"]])
def test_cli_argument_errors_exit_zero(args):
    assert _cli(*args).returncode == 0


def test_cli_missing_model_reports_an_error():
    p = _cli("-m", "/nonexistent/model.xml", "-q", "10", "10", "1", "1", "1", "0", "")
    assert p.returncode == 1
    assert "does not exist" in (p.stdout + p.stderr)
