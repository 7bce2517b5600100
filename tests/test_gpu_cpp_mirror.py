"""The C++ mirror (include/cpm.hpp) run on the GPU: reference cases through the C++ host side."""
import subprocess

import pytest

from test_abi import _compile_mirror

pytestmark = pytest.mark.gpu


def test_cpp_mirror_runs_reference_cases(cpm, tmp_path):
    from importlib import import_module
    native = import_module("cosmological-particle-simulation_b200._native")
    exe = _compile_mirror(native, tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all ok" in r.stdout
