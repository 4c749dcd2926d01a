import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and, when missing, the CUDA library (nvcc cross-compiles without a GPU)."""
    from oracle import oracle as O
    O.build()
    from onemirror_b200 import build as B
    if not os.path.exists(B.LIB):
        B.build()
    yield


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
