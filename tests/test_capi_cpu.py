"""C ABI checks that need no GPU: the library loads, exports every function
include/amss_b200.h declares, and fails loudly (no CPU fallback) when no CUDA
device is usable."""
import ctypes

import pytest
import torch

import amss_b200
from amss_b200 import _lib


def test_library_exports_every_header_function():
    L = amss_b200.lib()
    names = amss_b200.header_functions()
    assert "compute_rhs_bssn_" in names and "amss_engine_create" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in amss_b200.lib().amss_version()


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device failure path")
def test_engine_refuses_without_device():
    with pytest.raises(amss_b200.AmssError, match="no usable CUDA device"):
        amss_b200.Engine()


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device failure path")
def test_dropin_refuses_without_device():
    import numpy as np
    X = np.linspace(-1, 1, 8)
    st = np.zeros((24, 8, 8, 8))
    with pytest.raises(amss_b200.AmssError):
        amss_b200.dropin.compute_rhs_bssn(X, X, X, st)
