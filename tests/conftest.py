import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")

# Material of every parity case: E = 1e5 Pa, nu = 0.45.
E_YOUNG, NU = 1e5, 0.45


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name))
    return load


@pytest.fixture(scope="session")
def lib_built():
    """Build the CUDA library if needed (nvcc cross-compiles without a GPU)."""
    from wrapd_b200 import build
    return build.build()
