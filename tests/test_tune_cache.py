"""The autotuner's selection rule and its cache file (CPM_TUNE_CACHE) on the CPU: the host-only
header csrc/tune_cache.h that sim.cu uses, compiled with g++ into a small checker."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_tune_selection_and_cache_file(tmp_path):
    exe = tmp_path / "tune_cache_check"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror",
           "-I", str(ROOT / "cosmological-particle-simulation_b200" / "csrc"),
           str(ROOT / "tests" / "cpp" / "tune_cache_check.cpp"), "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe), str(tmp_path / "tune.txt")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    for part in ("selection ok", "line ok", "rejection ok", "file ok"):
        assert part in r.stdout
