"""Shared pytest set-up: the `gpu` marker, import paths, and the two libraries under test."""
import importlib
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def cpm():
    """The product package (ctypes front end of libcpm_cuda.so)."""
    return importlib.import_module("cosmological-particle-simulation_b200")
