import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "libnegf.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libnegf_b200.so")


@pytest.fixture(scope="session")
def negf():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import libnegf_b200
    libnegf_b200.load()
    return libnegf_b200


def rel_fro(a, b):
    import numpy as np
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)
