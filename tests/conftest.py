import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 and the built libbanana_b200.so")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def bnn():
    """The CUDA library; GPU tests fail (not skip) when it or the GPU is missing."""
    import torch
    import banana_b200 as B
    from banana_b200 import build as bld
    if not bld.LIB.exists():
        bld.build()
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    B.load()
    return B
