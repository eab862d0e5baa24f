"""Shared fixtures.  `-m gpu` tests need a CUDA device and the in-tree libwp_b200.so; the CPU suite
checks the oracle against the reference's golden fixtures, the host logic and the C ABI surface."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built libwp_b200.so")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def wp():
    """The product package on a GPU: fails loudly if the extension or the device is missing."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    from waveletpotentials_b200 import api, build
    build.build()
    return api
