"""Shared test setup: import paths, the ``gpu`` marker and fixtures.

``-m "not gpu"`` tests run anywhere (oracle vs golden vectors, host logic,
the C ABI loads and exports every declared symbol).  ``-m gpu`` tests call
the CUDA kernels through the C ABI and compare them with the oracle.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("cuda-n4_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built libn4b200.so")


@pytest.fixture(scope="session")
def golden_components():
    return np.load(os.path.join(GOLDEN, "components.npz"))


@pytest.fixture(scope="session")
def golden_small():
    return np.load(os.path.join(GOLDEN, "n4_small.npz"))


@pytest.fixture(scope="session")
def golden_c1():
    path = os.path.join(GOLDEN, "n4_c1.npz")
    if not os.path.exists(path):
        pytest.skip("n4_c1.npz not generated")
    return np.load(path)


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    import n4b200
    n4b200.library()
    return torch
