"""Moving boxes: the refined boxes follow the tracked punctures.

cgh::Regrid_Onelevel (cgh.C:1304-1506) checks, per moving level and per box
of that level (one box per puncture, cgh::bbox[lev][grd]), how far the
puncture (Porg0, tracked on the finest level) has moved from the box's
centre (its `handle`).  A box is matched to the puncture whose position at
the level's last regrid (Porgls) lies within 2 * do_every cells of the
centre (do_every = 2; with one puncture it always matches).  Per axis the
offset in cells is rounded half away from zero, truncated to a multiple of
do_every, and if that moves the box by more than half a cell the box and its
centre shift by it; Porgls of the puncture takes the new position on that
axis.  If any box of the level moved, the level is rebuilt
(recompose_cgh_Onelevel) and its data refilled (Parallel::fill_level_data):
cells the old level held are copied, new cells are prolonged from the parent
level -- in time too for the previous time level.

This engine checks every moving level at the end of a coarse step, when
every level sits at the same time, finest level first, each refill reading
the old engine (so a level's new cells come from its parent's old boxes, as
in the reference, where a level regrids at the end of its own RecursiveStep,
before its parent does).  The reference also checks a fine level at the end
of each of its RecursiveSteps inside a coarse step; here such a level moves
once per coarse step by the accumulated offset.
"""
import copy

import numpy as np

from .hierarchy import from_boxes

DO_EVERY = 2


def _c_int(x):
    """C's int() of a double: truncation toward zero."""
    return int(np.trunc(x))


class Regridder:
    """The moving-box state of a hierarchy built by from_boxes (box_in_box,
    the par-file front end): per level >= movls the unmerged boxes (global
    cells), their centres and Porgls."""

    def __init__(self, H, punctures, movls=1, symmetry=0):
        self.x0, self.h0 = H.x0, H.h0
        self.args = dict(H.build_args)
        self.movls = movls
        self.symmetry = symmetry
        self.boxes = copy.deepcopy(H.grid_boxes)          # levels 1..: list of [lo, hi]
        self.handles = [[self._centre(lv + 1, b) for b in bl] for lv, bl in enumerate(self.boxes)]
        self.porgls = [[list(map(float, p)) for p in punctures] for _ in self.boxes]

    def _centre(self, lev, box):
        h = self.h0 / 2 ** lev
        return [self.x0 + 0.5 * (box[0][d] + box[1][d]) * h for d in range(3)]

    def plan(self, porg0):
        """New boxes for the tracked positions porg0; returns the levels
        that move (finest first), and updates the state."""
        moved = []
        nbh = len(porg0)
        for lev in range(len(self.boxes), 0, -1):
            if lev < self.movls:
                continue
            li = lev - 1
            dX = self.h0 / 2 ** lev
            tmp = [list(p) for p in self.porgls[li]]
            tot = False
            for grd, box in enumerate(self.boxes[li]):
                handle = self.handles[li][grd]
                bhi = next((b for b in range(nbh)
                            if all(abs(self.porgls[li][b][d] - handle[d]) < 2 * DO_EVERY * dX for d in range(3))),
                           nbh)
                if bhi == nbh:
                    lo_phys = [self.x0 + box[0][d] * dX for d in range(3)]
                    if all(abs(0.0 - lo_phys[d]) < dX / 2 for d in range(3)):
                        break   # a box already at the origin (cgh.C:1370-1374)
                    if nbh == 1:
                        bhi = 0
                    else:
                        raise ValueError(f"regrid: no puncture matches level {lev} box {grd}")
                for d in range(3):
                    rr = (porg0[bhi][d] - handle[d]) / dX
                    flag = (_c_int(rr + 0.5) if rr > 0 else _c_int(rr - 0.5))
                    flag = int(flag / DO_EVERY) * DO_EVERY            # C integer division truncates
                    lo_new = self.x0 + box[0][d] * dX + flag * dX
                    if ((d < 2 and self.symmetry == 2) or (d == 2 and self.symmetry > 0)) and lo_new < 0:
                        raise ValueError("regrid: a box would cross a symmetry plane (not supported)")
                    if abs(flag * dX) > dX / 2:
                        tot = True
                        box[0][d] += flag
                        box[1][d] += flag
                        handle[d] += flag * dX
                        tmp[bhi][d] = porg0[bhi][d]
            if tot:
                moved.append(lev)
                self.porgls[li] = tmp
        return moved

    def hierarchy(self):
        a = self.args
        return from_boxes(self.x0, self.h0, a["coarse"], self.boxes, a["seed"], a["block_min"], a["block_max"])


def regrid(eng, H, regridder, porg0=None):
    """Apply the moving-box rule after a coarse step.  Returns (engine,
    hierarchy, moved levels): the same engine and hierarchy if nothing moved,
    else a new engine over the new hierarchy holding the refilled data (the
    old engine is closed), with the same tiling and puncture tracking."""
    if porg0 is None:
        porg0 = eng.punctures().tolist()
    moved = regridder.plan(porg0)
    if not moved:
        return eng, H, []
    H2 = regridder.hierarchy()
    from .engine import Engine
    eng.sync()
    new = Engine.from_hierarchy(H2, **eng.params)
    for lv in range(len(H2.levels)):
        for back in (0, 1):
            new.regrid_fill(eng, lv, back)
        w, z, _ = eng.level_tiling(lv)
        new.set_level_tiling(lv, w, z)
        new.set_level_occupancy(lv, eng.level_occupancy(lv))
    if getattr(eng, "_ntrack", 0):
        new.set_punctures(porg0)
    eng.close()
    return new, H2, moved
