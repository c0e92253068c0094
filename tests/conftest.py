import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def mesh():
    from cellsim3d_b200 import workloads as W
    return W.load_mesh()


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and the library in-tree if they are missing."""
    import oracle
    oracle.lib()
    from cellsim3d_b200 import build
    if not os.path.exists(build.LIB):
        build.build()
