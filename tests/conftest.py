import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def lemc():
    """The native library, built in-tree if needed."""
    from laughlinedge_b200 import build
    build.build()
    import laughlinedge_b200 as L
    L.load()
    return L


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.load()
    return O


@pytest.fixture(scope="session")
def cuda_ctx(lemc):
    """torch on cuda:0 for device buffers; fails loudly without a GPU."""
    import torch
    assert torch.cuda.is_available(), "GPU test collected on a machine without CUDA"
    torch.cuda.init()
    return torch
