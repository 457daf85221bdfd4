import os
import sys

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def pytest_collection_modifyitems(config, items):
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def rel(a, b):
    a = torch.as_tensor(a).to(torch.complex128) if torch.as_tensor(a).is_complex() else torch.as_tensor(a).double()
    b = torch.as_tensor(b).to(a.dtype)
    return float((a.cpu() - b.cpu()).norm() / b.cpu().norm().clamp_min(1e-300))


@pytest.fixture(scope="session")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mrirecon_b200._lib as L
    L.load()
    return torch.device("cuda", 0)
