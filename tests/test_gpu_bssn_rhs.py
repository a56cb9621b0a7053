"""GPU parity of the drop-in compute_rhs_bssn_ (C ABI) against the CPU oracle.

Bar: FP64, relative max-norm error per output field <= 1e-12 over all points
of the block (outer planes included)."""
import numpy as np
import pytest

import oracle as O
from amss_b200 import dropin as D

from helpers import generic_state, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _check(ref, got, tol=TOL):
    g_ref, r_ref = ref[0], ref[1:]
    g_got, r_got = got[0], got[1:]
    assert g_ref == g_got
    worst = {}
    for group, (a, b) in enumerate(zip(r_got, r_ref)):
        for f in range(a.shape[0]):
            worst[(group, f)] = relerr(a[f], b[f])
    bad = {k: v for k, v in worst.items() if v > tol}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])[:8]
    return max(worst.values())


def test_rhs_config1_block():
    """64^3 interior + 3 cells each side on [-8, 8]^3 (dx = 0.25), one
    Brill-Lindquist puncture m = 1 at (0.1, 0.05, 0.02), uniform noise 1e-8."""
    X, st, bbox, h = O.single_block_setup(64, -8.0, 8.0, 3, [1.0], [[0.1, 0.05, 0.02]], noise=1e-8, seed=1)
    ref = O.compute_rhs_bssn(X, X, X, st, eps=0.1, co=0)
    got = D.compute_rhs_bssn(X, X, X, st, eps=0.1, co=0)
    _check(ref, got)


@pytest.mark.parametrize("shape", [(20, 22, 24), (9, 13, 11)])
def test_rhs_generic_state(shape):
    """Every field non-zero, shift of both signs: exercises all lopsided
    branches, the 2nd-order boundary fallback and the KO gate."""
    nx, ny, nz = shape
    X = O.cell_coords(-2.0, 2.5, nx)
    Y = O.cell_coords(-1.5, 2.0, ny)
    Z = O.cell_coords(-3.0, 1.0, nz)
    st = generic_state(X, Y, Z, seed=7)
    rng = np.random.default_rng(11)
    matter = 1e-3 * rng.standard_normal((10, nz, ny, nx))
    ref = O.compute_rhs_bssn(X, Y, Z, st, matter=matter, eps=0.2, co=0)
    got = D.compute_rhs_bssn(X, Y, Z, st, matter=matter, eps=0.2, co=0)
    _check(ref, got)
    ref = O.compute_rhs_bssn(X, Y, Z, st, eps=0.0, co=1)
    got = D.compute_rhs_bssn(X, Y, Z, st, eps=0.0, co=1)
    _check(ref, got)


@pytest.mark.parametrize("symmetry", [1, 2])
def test_rhs_symmetry_planes(symmetry):
    """Blocks whose low faces sit on the symmetry planes (z = 0 for equatorial,
    x = y = z = 0 for octant) read the mirrored pad of symmetry_bd."""
    lo = 0.0 if symmetry == 2 else -2.0
    X = O.cell_coords(lo, 2.0, 14 if symmetry == 2 else 18)
    Y = O.cell_coords(lo, 2.0, 12 if symmetry == 2 else 16)
    Z = O.cell_coords(0.0, 2.0, 10)
    st = generic_state(X, Y, Z, seed=5)
    ref = O.compute_rhs_bssn(X, Y, Z, st, symmetry=symmetry, eps=0.1, co=0)
    got = D.compute_rhs_bssn(X, Y, Z, st, symmetry=symmetry, eps=0.1, co=0)
    _check(ref, got)


def test_rhs_nan_leaves_outputs_untouched():
    X = O.cell_coords(-1.0, 1.0, 10)
    st = generic_state(X, X, X)
    st[9][4, 5, 6] = np.nan
    gont, rhs, gam, ric, cons = D.compute_rhs_bssn(X, X, X, st, co=0)
    assert gont == 1 and np.all(rhs == 0) and np.all(cons == 0)
    st = generic_state(X, X, X)
    st[1][2, 2, 2] = np.inf
    st[2][3, 3, 3] = -np.inf
    assert D.compute_rhs_bssn(X, X, X, st)[0] == 1
    st = generic_state(X, X, X)
    st[21][2, 2, 2] = np.nan   # dtSfx is outside the reference's NaN check
    assert D.compute_rhs_bssn(X, X, X, st)[0] == 0
