"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    O.set_threads(0)
    return O


@pytest.fixture(scope="session")
def product():
    import ccpol23_plus_2025_mbmd_b200 as P
    from ccpol23_plus_2025_mbmd_b200 import build
    build.build()
    return P


def rel(a, b):
    """Normwise relative difference ||a - b|| / ||b|| (absolute when b is 0)."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    nb = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    return d / nb if nb > 0 else d
