"""The read reach of the transfer stencils that the engine's cell plans assume
(plan_final_regions and timeinterp_boxes in xfer.cu), checked against the
oracle's restatement of prolongrestrict_cell.f90.

* restrict3 of coarse cell k reads fine cells 2k-2 .. 2k+3 per axis;
* prolong3 of fine cell g reads coarse cells (g >> 1) - 3 .. (g >> 1) + 2 when
  g is even, (g >> 1) - 2 .. (g >> 1) + 3 when g is odd.

Every cell outside the assumed reach holds NaN, so a read past it would show;
every cell inside is read (a NaN planted there reaches the result)."""
import itertools

import numpy as np
import pytest

import oracle as O
from amr import _I3, _p


def _reach_prolong(g):
    c = g >> 1
    return (c - 3, c + 3) if g % 2 == 0 else (c - 2, c + 4)


def _box(n, lo, hi):
    a = np.full((n, n, n), np.nan)
    a[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] = 1.0
    return a


@pytest.mark.parametrize("k", [(4, 4, 4), (3, 5, 4)])
def test_restrict3_reads_fine_2k_minus_2_to_2k_plus_3(k):
    lib = O.lib()
    nf, nc = 16, 8
    lo = [2 * v - 2 for v in k]
    hi = [2 * v + 4 for v in k]
    fine = _box(nf, lo, hi)
    coarse = np.zeros((nc, nc, nc))
    lib.oracle_restrict3_box(_I3(nc, nc, nc), _I3(0, 0, 0), _p(coarse), _I3(nf, nf, nf), _I3(0, 0, 0), _p(fine),
                             _I3(*k), _I3(*[v + 1 for v in k]))
    got = coarse[k[2], k[1], k[0]]
    assert np.isfinite(got) and abs(got - 1.0) < 1e-14
    for corner in itertools.product(*[(lo[d], hi[d] - 1) for d in range(3)]):
        poisoned = fine.copy()
        poisoned[corner[2], corner[1], corner[0]] = np.nan
        c2 = np.zeros((nc, nc, nc))
        lib.oracle_restrict3_box(_I3(nc, nc, nc), _I3(0, 0, 0), _p(c2), _I3(nf, nf, nf), _I3(0, 0, 0), _p(poisoned),
                                 _I3(*k), _I3(*[v + 1 for v in k]))
        assert np.isnan(c2[k[2], k[1], k[0]])


@pytest.mark.parametrize("g", [(14, 14, 14), (15, 15, 15), (14, 15, 17)])
def test_prolong3_reads_the_parity_dependent_six_coarse_cells(g):
    lib = O.lib()
    nc, nf = 16, 32
    lo, hi = zip(*[_reach_prolong(v) for v in g])
    coarse = _box(nc, lo, hi)
    fine = np.zeros((nf, nf, nf))
    lib.oracle_prolong3_box(_I3(nc, nc, nc), _I3(0, 0, 0), _p(coarse), _I3(nf, nf, nf), _I3(0, 0, 0), _p(fine),
                            _I3(*g), _I3(*[v + 1 for v in g]))
    got = fine[g[2], g[1], g[0]]
    assert np.isfinite(got) and abs(got - 1.0) < 1e-14
    for corner in itertools.product(*[(lo[d], hi[d] - 1) for d in range(3)]):
        poisoned = coarse.copy()
        poisoned[corner[2], corner[1], corner[0]] = np.nan
        f2 = np.zeros((nf, nf, nf))
        lib.oracle_prolong3_box(_I3(nc, nc, nc), _I3(0, 0, 0), _p(poisoned), _I3(nf, nf, nf), _I3(0, 0, 0), _p(f2),
                                _I3(*g), _I3(*[v + 1 for v in g]))
        assert np.isnan(f2[g[2], g[1], g[0]])
