"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def built():
    """Builds the oracle and the CUDA library in-tree (nvcc cross-compiles without a GPU)."""
    from oracle import oracle
    from icoatmosbenchmark_v1_b200 import build
    oracle.build()
    if not os.environ.get("ICOADV_NO_BUILD"):
        build.build()
    return True


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    return torch.device("cuda:0")
