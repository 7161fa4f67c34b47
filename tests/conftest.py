import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size configurations")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def t213():
    return importlib.import_module("213transpose_b200")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch


def to_device(torch, host: np.ndarray):
    """Raw bytes -> uint8 CUDA tensor (element size is passed explicitly)."""
    return torch.from_numpy(host.view(np.uint8).copy()).cuda()


def from_device(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint8)
