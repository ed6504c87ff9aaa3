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


def kappa_tol(cond, tol=1e-12):
    """Parity bound between two FP64 inversions of the same matrix: each is
    backward stable with a normwise forward error near u * kappa (u = 2^-53),
    so they may differ by 2 u kappa. The 1e-12 bar stands up to kappa ~ 4.5e3;
    the stress generators also draw worse-conditioned matrices."""
    return max(tol, 2.0 * 2.0 ** -53 * float(cond))
