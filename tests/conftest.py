"""Shared pytest configuration.

Markers:
* ``gpu``  -- needs a CUDA device (B200, sm_100a); run with ``-m gpu``.
* ``slow`` -- long CPU cases, deselected by default runs of ``-m "not gpu"``
  only when ``-m "not slow"`` is also given.
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (sm_100a)")
    config.addinivalue_line("markers", "slow: long-running test")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "lbm_golden.npz")
    return np.load(path)
