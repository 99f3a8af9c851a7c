"""The C-ABI library loads and exports every symbol include/ccpol23_b200.h declares; without
a GPU, creating a context fails with CCP_ERR_NO_DEVICE (never a silent CPU fallback)."""
import ctypes as C
import re
from pathlib import Path

import pytest
import torch

from ccpol23_plus_2025_mbmd_b200 import CcpError, Context, Model, data_dir
from ccpol23_plus_2025_mbmd_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "ccpol23_b200.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(ccp_\w+)\s*\(", text)))


def test_header_and_binding_agree(product):
    assert declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_symbol(product):
    L = C.CDLL(str(_lib.LIB_PATH))
    for name in declared():
        assert hasattr(L, name), name


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU path")
def test_no_device_is_an_error(product):
    m = Model(data_dir("fs3"))
    with pytest.raises(CcpError) as e:
        Context(m, 128, 15.64)
    assert e.value.code == _lib.CCP_ERR_NO_DEVICE
