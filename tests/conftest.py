"""Shared fixtures.  Tests marked ``gpu`` need a B200 and the built
libelmm_gpu.so; everything else runs on the CPU (oracle, host logic, C-ABI
surface)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    yield


def rel(a, b):
    """max |a - b| / max |b| (1 if b is zero)."""
    import numpy as np
    s = float(np.abs(b).max())
    return float(np.abs(a - b).max()) / (s if s > 0 else 1.0)
