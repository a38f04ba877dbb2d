"""Shared pytest configuration.

``-m gpu`` tests run the CUDA library on a B200 and compare it with the oracle; everything else
runs on CPU (oracle pinning, host logic, C-ABI loading)."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running case")


def colmajor(X):
    """Column-major storage of a logical (m x n) torch matrix: an (n, m) contiguous tensor.
    Always a fresh copy (``.contiguous()`` alone aliases vectors and 1 x 1 matrices)."""
    import torch
    return X.t().clone(memory_format=torch.contiguous_format)


def logical(Xcm):
    """Logical matrix from its column-major storage tensor."""
    return Xcm.t()


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import cuev_b200
    cuev_b200.lib()
    return torch.device("cuda:0")
