"""The moving-box rule on CPU: the product's planner (amss_b200.regrid) against
the oracle's restatement of cgh::Regrid_Onelevel (oracle/amr.py) over seeded
puncture drifts, level by level, finest first."""
import copy

import numpy as np

from amss_b200.hierarchy import box_in_box
from amss_b200.regrid import Regridder
import amr as OA


def _oracle_plan(boxes, handles, porgls, porg0, x0, h0):
    moved = []
    for lev in range(len(boxes), 0, -1):
        m, porgls[lev - 1] = OA.regrid_onelevel(lev, boxes[lev - 1], handles[lev - 1], porgls[lev - 1], porg0, x0, h0)
        if m:
            moved.append(lev)
    return moved


def test_planner_matches_the_oracle_over_seeded_drifts():
    rng = np.random.default_rng(3)
    for centres in ([(1.2, 0.3, -0.4)], [(-3.0, 0.0, 0.0), (3.0, 0.0, 0.0)]):
        H = box_in_box(96, 48.0, centres, 6, box_cells=48, seed=1, block_min=18, block_max=74)
        r = Regridder(H, centres)
        boxes, handles = copy.deepcopy(r.boxes), copy.deepcopy(r.handles)
        porgls = [[list(p) for p in centres] for _ in boxes]
        pos = [list(p) for p in centres]
        for step in range(12):
            pos = [[p[d] + rng.uniform(-0.08, 0.08) for d in range(3)] for p in pos]
            got = r.plan(pos)
            want = _oracle_plan(boxes, handles, porgls, pos, H.x0, H.h0)
            assert got == want, step
            assert r.boxes == boxes and np.allclose(r.handles, handles) and r.porgls == porgls, step
        H2 = r.hierarchy()
        assert len(H2.levels) == len(H.levels)


def test_planner_moves_by_even_cells():
    H = box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    r = Regridder(H, [(1.2, 0.3, -0.4)])
    lo1, lo2 = list(r.boxes[0][0][0]), list(r.boxes[1][0][0])
    assert r.plan([(1.75, 0.3, -0.4)]) == [2, 1]
    assert r.boxes[1][0][0][0] - lo2[0] == 4 and r.boxes[0][0][0][0] - lo1[0] == 2
    assert r.boxes[1][0][0][1:] == lo2[1:]
    assert r.plan([(1.75, 0.3, -0.4)]) == []   # nothing left to move
