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


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device failure path")
def test_adjoint_and_initial_data_refuse_without_device():
    import numpy as np
    with pytest.raises(amss_b200.AmssError, match="no usable CUDA device"):
        amss_b200.adjoint.Adjoint((12, 12, 12), (-1, -1, -1, 1, 1, 1))
    X = np.linspace(-1, 1, 8)
    with pytest.raises(amss_b200.AmssError):
        amss_b200.dropin.get_lousto_nbhs(X, X, X, [1.0], [[0.1, 0.0, 0.0]])


def test_product_noise_equals_the_oracles():
    """Bench inputs (amss_b200.initial) and test inputs (the oracle) draw the
    same per-cell noise."""
    import numpy as np
    import amr as OA
    from amss_b200 import initial
    rng = np.random.default_rng(0)
    gi, gj, gk = (rng.integers(-500, 70000, 2000) for _ in range(3))
    for level, field, seed in [(0, 0, 1), (5, 23, 7), (7, 24, 123456789)]:
        a = initial.grid_noise(level, field, gi, gj, gk, seed)
        b = OA.grid_noise(level, field, gi, gj, gk, seed)
        assert np.array_equal(a, b)
        assert a.min() >= -1.0 and a.max() < 1.0
