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
    """Build the oracle (and the CUDA library, when nvcc is present) once."""
    from oracle import oracle as orc
    orc.build()
    try:
        from lceqcd_b200 import build as b
        b.build()
    except RuntimeError as e:  # no nvcc: only the oracle tests can run
        print("lceqcd_b200 build skipped:", e)
    yield


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
