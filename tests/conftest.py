"""Shared fixtures.  ``-m gpu`` tests need a CUDA device and the built libbs_b200.so; the rest run on CPU."""
import os
import sys
from dataclasses import dataclass

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


# The reference's own settings types as a caller holds them (src/openfawe/aero/vortex.py:30-116): the same field names
# and defaults and nothing more (no ``tree`` field, orders 0-2), for tests of what an unchanged caller reaches.
@dataclass(frozen=True)
class ReferenceTreeSettings:
    theta: float = 0.5
    order: int = 2
    leaf_size: int = 32
    core_clearance: float = 3.0

    def __post_init__(self):
        if self.order not in (0, 1, 2):
            raise ValueError("tree order must be 0, 1 or 2")


@dataclass(frozen=True)
class ReferenceCudaSettings:
    precision: str = "mixed"
    block: int = 128
    suspect: str = "cpu"
    control: str = "cpu"
    moments: str = "cpu"
    build: str = "cpu"
    rings: str = "cpu"
