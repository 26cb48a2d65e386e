"""Shared fixtures.  ``-m gpu`` tests need a CUDA device and the built libbs_b200.so; the rest run on CPU."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libbs_b200.so")


def golden(name):
    """A committed fixture made by tests/golden/make_golden.py from the reference's own code."""
    return np.load(os.path.join(GOLDEN, name))


def no_exclusions(n):
    return np.zeros(n + 1, dtype=np.int64), np.zeros(0, dtype=np.int64)


@pytest.fixture(scope="session")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.cuda.current_device()
