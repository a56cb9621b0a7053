"""GPU parity of the Z4c path against the CPU oracle (Z4c_rhs.f90:126-1295).

* compute_rhs_z4c_ (drop-in, FP64): right-hand sides and the diagnostic
  outputs on a Brill-Lindquist block and on generic states with Theta != 0,
  relative max-norm per field <= 1e-12;
* the engine with formulation="z4c" (split kernels): RK4 steps of a single
  block and Berger-Oliger coarse steps of a three-level hierarchy, FP64 bar
  1e-12, mixed bar 1e-6.
"""
import numpy as np
import pytest

import amss_b200
import amr as OA
import oracle as O
from amss_b200 import dropin as D
from amss_b200.hierarchy import box_in_box, single_block

from helpers import generic_state, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _theta(X, Y, Z, amp=2e-3):
    z, y, x = np.meshgrid(Z, Y, X, indexing="ij")
    return amp * np.sin(0.7 * x + 0.2) * np.cos(0.5 * y) * np.sin(0.9 * z + 0.4)


def _check(ref, got, tol=TOL):
    assert ref[0] == got[0]
    worst = {}
    for group, (a, b) in enumerate(zip(got[1:], ref[1:])):
        for f in range(a.shape[0]):
            worst[(group, f)] = relerr(a[f], b[f])
    bad = {k: v for k, v in worst.items() if v > tol}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])[:8]


def test_z4c_rhs_brill_lindquist_block():
    X, st, bbox, h = O.single_block_setup(40, -8.0, 8.0, 3, [1.0], [[0.1, 0.05, 0.02]], noise=1e-8, seed=1)
    st = np.concatenate([st, 1e-8 * np.random.default_rng(2).uniform(-1, 1, (1,) + st.shape[1:])])
    _check(O.compute_rhs_z4c(X, X, X, st, eps=0.1), D.compute_rhs_z4c(X, X, X, st, eps=0.1))


@pytest.mark.parametrize("shape", [(20, 22, 24), (9, 13, 11)])
def test_z4c_rhs_generic_state(shape):
    nx, ny, nz = shape
    X = O.cell_coords(-2.0, 2.5, nx)
    Y = O.cell_coords(-1.5, 2.0, ny)
    Z = O.cell_coords(-3.0, 1.0, nz)
    st = generic_state(X, Y, Z, seed=7)
    st = np.concatenate([st, _theta(X, Y, Z)[None]])
    matter = 1e-3 * np.random.default_rng(11).standard_normal((10, nz, ny, nx))
    _check(O.compute_rhs_z4c(X, Y, Z, st, matter=matter, eps=0.2),
           D.compute_rhs_z4c(X, Y, Z, st, matter=matter, eps=0.2))


@pytest.mark.parametrize("symmetry", [1, 2])
def test_z4c_rhs_symmetry_planes(symmetry):
    X = O.cell_coords(0.0, 2.0, 14) if symmetry == 2 else O.cell_coords(-2.0, 2.0, 14)
    Z = O.cell_coords(0.0, 2.0, 12)
    st = generic_state(X, X, Z, seed=5)
    st = np.concatenate([st, _theta(X, X, Z)[None]])
    _check(O.compute_rhs_z4c(X, X, Z, st, symmetry=symmetry, eps=0.1),
           D.compute_rhs_z4c(X, X, Z, st, symmetry=symmetry, eps=0.1))


def test_z4c_rhs_nan_in_theta():
    X = O.cell_coords(-2.0, 2.0, 10)
    st = np.zeros((25, 10, 10, 10))
    st[24, 5, 5, 5] = np.nan
    assert D.compute_rhs_z4c(X, X, X, st)[0] == 1


def _errs(got, ref):
    nf = ref[0].shape[0]
    errs = np.zeros(nf)
    for f in range(nf):
        den = max(max(np.abs(r[f]).max() for r in ref), 1e-300)
        errs[f] = max(np.abs(g[f] - r[f]).max() for g, r in zip(got, ref)) / den
    return errs


def _evolve(H, init, dt0, steps, precision="fp64"):
    oh = OA.OracleHierarchy(H, eps=0.1, nf=25)
    for i, st in enumerate(init):
        oh.set_state(i, st)
    for _ in range(steps):
        assert oh.coarse_step(dt0) == 0
    ref = [oh.state(i).copy() for i in range(len(H.blocks))]
    e = amss_b200.Engine.from_hierarchy(H, precision=precision, eps=0.1, formulation="z4c")
    for i, st in enumerate(init):
        e.set_state(i, st)
    for _ in range(steps):
        e.coarse_step(dt0)
    assert e.sync() == 0
    got = [e.get_state(i) for i in range(len(H.blocks))]
    e.close()
    return _errs(got, ref)


def _single(noise):
    H = single_block(24, -6.0, 6.0, 3)
    init = OA.initial_state(H, [1.0], [[0.1, 0.05, 0.02]], noise=noise, nf=25)
    return H, init, 0.25 * H.h0


@pytest.fixture(scope="module")
def single():
    return _single(1e-6)


def test_z4c_engine_single_block_fp64(single):
    H, init, dt0 = single
    errs = _evolve(H, init, dt0, 3)
    assert errs.max() <= TOL, errs


def test_z4c_engine_single_block_mixed():
    """Mixed bar on the Brill-Lindquist block with the BSSN tests' 1e-8 noise
    (FP32 stages carry g = d + 1 with ~6e-8 absolute rounding)."""
    H, init, dt0 = _single(1e-8)
    errs = _evolve(H, init, dt0, 3, precision="mixed")
    assert errs.max() <= 1e-6, errs


def test_z4c_engine_amr_fp64():
    H = box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-8, nf=25)
    errs = _evolve(H, init, 0.25 * H.h0, 1)
    assert errs.max() <= TOL, errs


def test_z4c_engine_rejects_wrong_state_shape(single):
    H, init, dt0 = single
    e = amss_b200.Engine.from_hierarchy(H, formulation="z4c")
    with pytest.raises(amss_b200._lib.AmssError):
        e.set_state(0, init[0][:24])
    e.close()
