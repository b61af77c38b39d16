import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product kernels")
    config.addinivalue_line("markers", "slow: long-running full-size case")


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def quest():
    """The libdgq QuEST API mirror, with one environment for the session."""
    if not have_gpu():
        pytest.skip("no CUDA device")
    from dgquest_b200 import quest as Q
    return Q


@pytest.fixture(scope="session")
def env(quest):
    e = quest.createQuESTEnv()
    yield e
    quest.destroyQuESTEnv(e)
