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


@pytest.mark.gpu
def test_noalloc_against_oracle_symmetry_and_matter():
    """Against the oracle (<= 1e-12 relative per output field): a block whose
    low z face sits on the equatorial plane (Symmetry 1, mirrored pads) with
    non-zero matter sources, then a block with no symmetry; two calls in a
    row through the shared static array."""
    import amss_b200
    from helpers import relerr
    rng = np.random.default_rng(17)
    X = O.cell_coords(-1.5, 1.5, 16)
    Z = O.cell_coords(0.0, 1.5, 12)
    st = generic_state(X, X, Z, seed=9)
    matter = 1e-3 * rng.standard_normal((10, 12, 16, 16))
    X2, st2 = _block(18, 4)
    cases = [(X, X, Z, st, matter, 1), (X2, X2, X2, st2, None, 0)]
    for Xc, Yc, Zc, s, m, sym in cases:
        ref = O.compute_rhs_bssn(Xc, Yc, Zc, s, matter=m, symmetry=sym, eps=0.1, co=0)
        got = amss_b200.dropin.compute_rhs_bssn_noalloc(Xc, Yc, Zc, s, matter=m, symmetry=sym, eps=0.1, co=0)
        assert ref[0] == got[0] == 0
        for r, g in zip(ref[1:], got[1:]):
            for f in range(r.shape[0]):
                assert relerr(g[f], r[f]) <= 1e-12, (sym, f)
