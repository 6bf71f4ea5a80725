"""Shared test configuration.

Tests marked ``gpu`` need a CUDA device and the built libcdgpu.so; everything
else runs on the CPU (oracle against the reference's golden fixtures, host
logic, library loading).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu)")


def golden(name):
    import refdump
    return refdump.load_npz(os.path.join(GOLDEN, name + ".npz"))


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle
