"""Results do not depend on how the patches are cut into blocks.

The reference cuts each patch into blocks by Parallel::distribute
(Parallel.C:504-827: near-equal pieces per axis, one per MPI rank); the
engine's hierarchies use seeded uneven cuts.  Every owned cell is computed by
the same arithmetic from the same values whatever the cut (the 3-cell ghost
zones carry the neighbours' owned values, the restriction and prolongation
read synchronised arrays), so the assembled patch data after two coarse steps
must be bit for bit the same for three different cuts of the same patches:
two seeded uneven splits and a split into near-equal halves per axis, as
distribute's pieces (with even cut points, which the engine needs so that no
coarse cell's children straddle two blocks)."""
import numpy as np
import pytest

import amss_b200
from amss_b200.hierarchy import Hierarchy, box_in_box, BUFFER
from amss_b200.io import patch_array
import amr as OA

pytestmark = pytest.mark.gpu


def _halves(lo, hi, parts=2):
    return [lo + (((hi - lo) * k // parts) & ~1) for k in range(1, parts)]


def _even_split_like(H0):
    """The same patches as H0, every patch (with its buffer) cut into 2 near-equal
    pieces per axis."""
    H = Hierarchy(H0.x0, H0.h0)
    for lev, patches in enumerate(H0.levels):
        for p in patches:
            elo, ehi = p.ext_lo, p.ext_hi
            H.add_patch(lev, p.lo, p.hi, p.buffer, [_halves(elo[d], ehi[d]) for d in range(3)])
    return H


def _run(H, steps=2):
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-8)
    e = amss_b200.Engine.from_hierarchy(H, eps=0.1)
    try:
        for i, st in enumerate(init):
            e.set_state(i, st)
        for _ in range(steps):
            e.coarse_step(0.25 * H.h0)
        assert e.sync() == 0
        st = [e.get_state(i) for i in range(len(H.blocks))]
    finally:
        e.close()
    return {(lv, pid): patch_array(H, lv, pid, lambda bi: st[bi])
            for lv in range(len(H.levels)) for pid in range(len(H.levels[lv]))}


def test_block_split_does_not_change_the_result():
    Ha = box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    Hb = box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=11, block_min=14, block_max=28)
    Hc = _even_split_like(Ha)
    assert BUFFER == 6
    cuts = [sorted(tuple(b.own_lo) for b in H.blocks) for H in (Ha, Hb, Hc)]
    assert cuts[0] != cuts[1] and cuts[0] != cuts[2]
    ra, rb, rc = _run(Ha), _run(Hb), _run(Hc)
    for key in ra:
        assert np.array_equal(ra[key], rb[key]), key
        assert np.array_equal(ra[key], rc[key]), key
