"""Argument checks of the Python API (no GPU needed): arrays that the library would read or
write out of bounds through raw pointers are refused with ValueError before any call into
it."""
import numpy as np
import pytest

from ccpol23_plus_2025_mbmd_b200 import Model, data_dir
from ccpol23_plus_2025_mbmd_b200._lib import ptr
from ccpol23_plus_2025_mbmd_b200.api import kspace_ewald_fixed


def test_numpy_pointer_refuses_wrong_arrays(product):
    assert ptr(None) is None
    assert ptr(np.zeros(3)) is not None
    with pytest.raises(ValueError):
        ptr(np.zeros(3, dtype=np.float32))
    with pytest.raises(ValueError):
        ptr(np.zeros((3, 4))[:, 1])
    with pytest.raises(ValueError):
        ptr([0.0, 1.0])


def test_fixed_scratch_refuses_host_and_misshaped_tensors(product):
    import torch
    m = Model(data_dir("fs3"))
    nm, ld = 4, 28
    mol = [torch.zeros(nm, dtype=torch.float64) for _ in range(3)]
    site = [torch.zeros(nm, ld, dtype=torch.float64) for _ in range(6)]
    one = [torch.zeros(1, dtype=torch.float64) for _ in range(2)]
    with pytest.raises(ValueError, match="CUDA"):
        kspace_ewald_fixed(m, *mol, *site[:3], 5, 5, 5, 0.35, 12.0, one[0], *site[3:], one[1])
    with pytest.raises(ValueError, match="ld"):
        short = [torch.zeros(nm, 3, dtype=torch.float64) for _ in range(3)]
        kspace_ewald_fixed(m, *mol, *short, 5, 5, 5, 0.35, 12.0, one[0], *site[3:], one[1])
