import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and the in-tree libraries if a fresh checkout lacks them."""
    import oracle
    from ampcor_b200 import build

    oracle.load()
    if not os.path.exists(build.SYNTH):
        build.build()
    yield


def cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
