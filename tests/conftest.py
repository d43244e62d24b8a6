"""Shared test configuration.

Markers: ``gpu`` -- needs a CUDA device (run with ``-m gpu`` on a B200);
everything else runs on CPU (``-m "not gpu"``).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def restatement():
    """The plain-C oracle (built on demand)."""
    from oracle import refcase as R
    if not os.path.exists(R.LIB_PATH):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       stdout=subprocess.DEVNULL)
    return R.Restatement()


@pytest.fixture(scope="session")
def golden_steps():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "steps.npz"))
