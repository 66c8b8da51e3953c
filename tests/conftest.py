import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libknnsweet.so")


def pytest_sessionstart(session):
    """Build the library and the command line in-tree when they are missing
    (nvcc cross-compiles without a GPU)."""
    from knn_sweet_b200 import build as kb
    if not kb.LIB.exists() or not kb.CLI.exists():
        kb.build()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.load()
    return o


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
