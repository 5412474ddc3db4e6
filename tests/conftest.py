"""Test configuration: the `gpu` marker and shared fixtures.

CPU tests (-m "not gpu") check the oracle against the reference's golden
vectors and the C ABI library's exports.  GPU tests (-m gpu) call the CUDA
library through its C ABI and compare against the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    return dict(np.load(os.path.join(ROOT, "tests", "golden", "reference_golden.npz")))


@pytest.fixture(scope="session")
def rlib():
    """The CUDA library; built if missing.  There is no CPU fallback."""
    import raptr_b200
    from raptr_b200 import build

    build.build()
    return raptr_b200
