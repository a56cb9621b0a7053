"""amss_compute_rhs_bssn_noalloc: compute_rhs_bssn_ with its device staging in
a static array of the library instead of cudaMalloc'd memory.

Collected last on purpose, so that it also runs after every other GPU test has
used the device (and the allocating drop-ins have grown their buffers)."""
import numpy as np
import pytest

import oracle as O

from helpers import generic_state


def _block(n, seed):
    X = O.cell_coords(-2.0, 2.0, n)
    st = generic_state(X, X, X, seed)
    return X, st


def test_noalloc_rejects_oversized_block():
    """Blocks over the static limit fail with AMSS_ERR_ARG before any device work."""
    import amss_b200
    from amss_b200._lib import AmssError
    X = O.cell_coords(-2.0, 2.0, 33)           # 33^3 = 35937 > 32768 points
    st = np.zeros((24, 33, 33, 33))
    with pytest.raises(AmssError, match="static scratch limit of 32768 points"):
        amss_b200.dropin.compute_rhs_bssn_noalloc(X, X, X, st)


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_twice():
    """Two calls in a row, different blocks and sizes: each output equals the
    allocating entry point's bit for bit (same kernel, same inputs)."""
    import amss_b200
    for n, seed, co in ((20, 3, 0), (14, 5, 1)):
        X, st = _block(n, seed)
        ref = amss_b200.dropin.compute_rhs_bssn(X, X, X, st, eps=0.1, co=co)
        got = amss_b200.dropin.compute_rhs_bssn_noalloc(X, X, X, st, eps=0.1, co=co)
        assert ref[0] == got[0] == 0
        for r, g in zip(ref[1:], got[1:]):
            assert np.array_equal(r, g)
