import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100) and the built CUDA library")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle

    pyoracle.load_port()
    return pyoracle


@pytest.fixture(scope="session")
def bf():
    """The CUDA backend; GPU tests fail (never skip) when it cannot run."""
    import batchfit_b200

    assert batchfit_b200.cuda_available(), "GPU tests require an sm_100 device and the built library"
    return batchfit_b200


def rng(seed):
    return np.random.default_rng(seed)
