"""Moving-box regrid on the GPU against the oracle: after two coarse steps of
a three-level hierarchy the tracked puncture is displaced (by 0.55 in x, as
a few coarse steps of an inspiral would), both refined levels move
(amss_b200.regrid: the box rule, a new engine, amss_engine_regrid_fill for the
current and previous time levels), and the refilled hierarchy must equal the
oracle's refill (oracle/amr.py: regrid_onelevel, OracleHierarchy.regrid_fill)
-- and still after one more coarse step, which reads the previous time levels
through the parent's time interpolation -- to <= 1e-12 per field."""
import copy

import numpy as np
import pytest

import amss_b200
from amss_b200.hierarchy import box_in_box
from amss_b200.regrid import Regridder, regrid
import amr as OA

pytestmark = pytest.mark.gpu

POS = [[1.2, 0.3, -0.4]]
DRIFT = [[1.75, 0.3, -0.4]]


def _errs(got, ref):
    errs = np.zeros(24)
    for f in range(24):
        den = max(max(np.abs(r[f]).max() for r in ref), 1e-300)
        errs[f] = max(np.abs(g[f] - r[f]).max() for g, r in zip(got, ref)) / den
    return errs


@pytest.mark.parametrize("precision", ["fp64"])
def test_regrid_matches_the_oracle(precision):
    H = box_in_box(40, 10.0, [tuple(POS[0])], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    init = OA.initial_state(H, [1.0], POS, noise=1e-8)
    dt0 = 0.25 * H.h0
    e = amss_b200.Engine.from_hierarchy(H, precision=precision, eps=0.1)
    oh = OA.OracleHierarchy(H, eps=0.1)
    for i, st in enumerate(init):
        e.set_state(i, st)
        oh.set_state(i, st)
    e.set_punctures(POS)
    oh.set_punctures(POS)
    for _ in range(2):
        e.coarse_step(dt0)
        assert oh.coarse_step(dt0) == 0
    assert e.sync() == 0

    r = Regridder(H, POS)
    boxes, handles = copy.deepcopy(r.boxes), copy.deepcopy(r.handles)
    porgls = [[list(p) for p in POS] for _ in boxes]
    e2, H2, moved = regrid(e, H, r, porg0=DRIFT)
    assert moved == [2, 1]
    # the oracle's box move and refill
    for lev in (2, 1):
        m, porgls[lev - 1] = OA.regrid_onelevel(lev, boxes[lev - 1], handles[lev - 1], porgls[lev - 1], DRIFT,
                                                H.x0, H.h0)
        assert m
    assert boxes == r.boxes
    oh2 = OA.OracleHierarchy(H2, eps=0.1)
    for lv in range(len(H2.levels)):
        for back in (0, 1):
            oh2.regrid_fill(oh, lv, back)
    got = [e2.get_state(i) for i in range(len(H2.blocks))]
    ref = [oh2.state(i) for i in range(len(H2.blocks))]
    errs = _errs(got, ref)
    assert errs.max() <= 1e-12, errs
    # one more coarse step from the refilled hierarchy
    oh2.set_punctures(DRIFT)
    e2.coarse_step(dt0)
    assert e2.sync() == 0
    assert oh2.coarse_step(dt0) == 0
    got = [e2.get_state(i) for i in range(len(H2.blocks))]
    ref = [oh2.state(i) for i in range(len(H2.blocks))]
    errs = _errs(got, ref)
    assert errs.max() <= 1e-12, errs
    assert np.array_equal(e2.punctures(), np.asarray(oh2.porg0))
    e2.close()


def test_regrid_refuses_unnested_boxes():
    """A move too large for the old parent level to cover fails cleanly."""
    H = box_in_box(40, 10.0, [tuple(POS[0])], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    init = OA.initial_state(H, [1.0], POS, noise=1e-8)
    e = amss_b200.Engine.from_hierarchy(H, precision="fp64", eps=0.1)
    for i, st in enumerate(init):
        e.set_state(i, st)
    r = Regridder(H, POS)
    r.boxes[1][0][0][0] += 40    # the finest box far beyond its parent
    r.boxes[1][0][1][0] += 40
    with pytest.raises(Exception):
        H2 = r.hierarchy()       # nesting check, before any device work
        e2 = amss_b200.Engine.from_hierarchy(H2, **e.params)
        e2.regrid_fill(e, 2, 0)
    e.close()
