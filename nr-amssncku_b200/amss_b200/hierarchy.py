"""Grid hierarchy description: levels -> patches -> blocks.

A static restatement of what the reference's cgh / Patch / Parallel::distribute
build (cgh.C:1212-1229 box merging, MPatch.C:14-190 buffer cells,
Parallel.C:504-827 block split with ghost cells), reduced to the pieces the
evolution path needs:

* Level l has cell size h0 / 2^l and a global cell index space whose cell I
  covers [x0 + I h_l, x0 + (I+1) h_l); coarse cell k has the fine children 2k
  and 2k+1.
* A patch is a box of cells [lo, hi) (its physical region); on levels > 0 it is
  extended by `buffer` cells (buffer_width = 6) on every side, filled by
  prolongation from the parent level after each step.
* A patch's extended box is split into blocks; a block's array is its owned
  box plus `ghost` cells (ghost_width = 3) on every side that faces another
  block of the same patch.  Split points are even so coarse cells are never
  split between blocks.

Coordinates follow Block.C:48-52 (Cell): X[j] = bbox_lo + (j + 0.5) h.
"""
from dataclasses import dataclass, field

import numpy as np

GHOST = 3
BUFFER = 6


@dataclass
class Patch:
    level: int
    lo: tuple          # physical box, global level indices [lo, hi)
    hi: tuple
    buffer: int
    blocks: list = field(default_factory=list)

    @property
    def ext_lo(self):
        return tuple(v - self.buffer for v in self.lo)

    @property
    def ext_hi(self):
        return tuple(v + self.buffer for v in self.hi)


@dataclass
class Block:
    level: int
    patch: int         # index of the patch within its level
    own_lo: tuple      # owned box, global level indices
    own_hi: tuple
    org: tuple         # global index of array element 0
    ex: tuple          # array extent


class Hierarchy:
    def __init__(self, x0, h0):
        self.x0 = float(x0)
        self.h0 = float(h0)
        self.levels = []   # list of lists of Patch
        self.blocks = []   # flat list of Block, in level order

    def h(self, level):
        return self.h0 / (2 ** level)

    def add_patch(self, level, lo, hi, buffer, splits):
        """splits: per axis the interior split points (global indices, even)."""
        while len(self.levels) <= level:
            self.levels.append([])
        p = Patch(level, tuple(lo), tuple(hi), buffer)
        pid = len(self.levels[level])
        self.levels[level].append(p)
        elo, ehi = p.ext_lo, p.ext_hi
        cuts = [[elo[d]] + sorted(splits[d]) + [ehi[d]] for d in range(3)]
        for k in range(len(cuts[2]) - 1):
            for j in range(len(cuts[1]) - 1):
                for i in range(len(cuts[0]) - 1):
                    olo = (cuts[0][i], cuts[1][j], cuts[2][k])
                    ohi = (cuts[0][i + 1], cuts[1][j + 1], cuts[2][k + 1])
                    alo = tuple(olo[d] - (GHOST if olo[d] > elo[d] else 0) for d in range(3))
                    ahi = tuple(ohi[d] + (GHOST if ohi[d] < ehi[d] else 0) for d in range(3))
                    b = Block(level, pid, olo, ohi, alo, tuple(ahi[d] - alo[d] for d in range(3)))
                    p.blocks.append(len(self.blocks))
                    self.blocks.append(b)
        return pid

    # coordinates ------------------------------------------------------------
    def bbox(self, b):
        h = self.h(b.level)
        return tuple(self.x0 + b.org[d] * h for d in range(3)) + \
            tuple(self.x0 + (b.org[d] + b.ex[d]) * h for d in range(3))

    def patch_bbox(self, p):
        h = self.h(p.level)
        return tuple(self.x0 + p.ext_lo[d] * h for d in range(3)) + tuple(self.x0 + p.ext_hi[d] * h for d in range(3))

    def phys_bbox(self, p):
        h = self.h(p.level)
        return tuple(self.x0 + p.lo[d] * h for d in range(3)) + tuple(self.x0 + p.hi[d] * h for d in range(3))

    def coords(self, b):
        """Block.C:48-52: X[j] = bbox_lo + (j + 0.5) * (bbox_hi - bbox_lo) / ex."""
        bb = self.bbox(b)
        out = []
        for d in range(3):
            h = (bb[3 + d] - bb[d]) / b.ex[d]
            out.append(np.array([bb[d] + (j + 0.5) * h for j in range(b.ex[d])]))
        return out

    def interior_zones(self, level):
        return sum(int(np.prod([p.hi[d] - p.lo[d] for d in range(3)])) for p in self.levels[level])

    def points(self, level):
        return sum(int(np.prod(self.blocks[i].ex)) for p in self.levels[level] for i in p.blocks)


def _splits(lo, hi, rng, min_pts, max_pts):
    """Seeded uneven even-index split points of [lo, hi) into pieces of
    min_pts..max_pts cells (the last piece takes the remainder)."""
    cuts = []
    x = lo
    while hi - x > max_pts:
        w = int(rng.integers(min_pts // 2, max_pts // 2 + 1)) * 2
        w = min(w, hi - x - min_pts)
        if w < min_pts:
            break
        x += w
        cuts.append(x)
    return cuts


def single_block(n_interior, lo, hi, ghosts=3):
    """One block that is the whole level-0 patch: n_interior cells on [lo, hi]
    plus `ghosts` cells each side, treated as ordinary evolved cells."""
    h = (hi - lo) / n_interior
    n = n_interior + 2 * ghosts
    H = Hierarchy(lo - ghosts * h, h)
    H.add_patch(0, (0, 0, 0), (n, n, n), 0, [[], [], []])
    return H


def merge_boxes(boxes, buffer=BUFFER):
    """Merge the boxes [lo, hi) of one level whose buffered extents meet into
    their bounding box, until no two meet.  The reference merges boxes that
    touch or overlap into their bounding box when that box is filled well
    enough (Parallel::merge_gs, Parallel.C:4997-5086) and cuts the others
    apart (cut_gsl); patches of this engine may not touch even through their
    buffers, so any two whose buffered boxes meet are merged."""
    boxes = [[list(lo), list(hi)] for lo, hi in boxes]
    merged = True
    while merged:
        merged = False
        for a in range(len(boxes)):
            for b in range(a + 1, len(boxes)):
                A, B = boxes[a], boxes[b]
                if all(A[0][d] - buffer <= B[1][d] + buffer and B[0][d] - buffer <= A[1][d] + buffer
                       for d in range(3)):
                    boxes[a] = [[min(A[0][d], B[0][d]) for d in range(3)], [max(A[1][d], B[1][d]) for d in range(3)]]
                    del boxes[b]
                    merged = True
                    break
            if merged:
                break
    return boxes


def from_boxes(x0, h0, coarse, levels, seed=1, block_min=24, block_max=80):
    """A hierarchy with the level-0 patch [0, coarse) (cells per axis) and, for
    levels 1.., the boxes levels[l - 1] (lists of [lo, hi) in that level's
    global cells), merged as merge_boxes does; every patch is split into seeded
    uneven blocks of block_min..block_max cells per side."""
    rng = np.random.default_rng(seed)
    coarse = tuple(coarse) if np.ndim(coarse) else (int(coarse),) * 3
    H = Hierarchy(x0, h0)
    # what a regrid rebuilds from: the boxes per level before merging (one per
    # puncture, as the reference keeps cgh::bbox per grid) and the split rule
    H.grid_boxes = [[[list(lo), list(hi)] for lo, hi in boxes] for boxes in levels]
    H.build_args = dict(coarse=coarse, seed=seed, block_min=block_min, block_max=block_max)
    H.add_patch(0, (0, 0, 0), coarse, 0, [_splits(0, coarse[d], rng, block_min, block_max) for d in range(3)])
    for lev, boxes in enumerate(levels, start=1):
        for lo, hi in merge_boxes(boxes):
            H.add_patch(lev, lo, hi, BUFFER,
                        [_splits(lo[d] - BUFFER, hi[d] + BUFFER, rng, block_min, block_max) for d in range(3)])
    H.check_nesting()
    return H


def box_in_box(coarse_cells, extent, centres, nlevels, box_cells=48, seed=1, block_min=24, block_max=80):
    """Config-2 style hierarchy: level 0 covers [-extent, extent]^3 with
    coarse_cells per side; levels 1..nlevels-1 carry one box of box_cells per
    side (in that level's cells) around each centre, boxes whose buffered
    extents overlap merged into their bounding box; every patch is split into
    seeded uneven blocks of block_min..block_max cells per side."""
    h0 = 2.0 * extent / coarse_cells
    x0 = -extent
    levels = []
    for lev in range(1, nlevels):
        h = h0 / 2 ** lev
        boxes = []
        for c in centres:
            lo = []
            for d in range(3):
                ci = int(round((c[d] - x0) / h))
                l0 = ci - box_cells // 2
                lo.append(l0 - (l0 % 2))
            boxes.append([lo, [v + box_cells for v in lo]])
        levels.append(boxes)
    return from_boxes(x0, h0, coarse_cells, levels, seed, block_min, block_max)


def _check(cond, msg):
    if not cond:
        raise ValueError(msg)


def _hierarchy_check(self):
    """Every refined patch (with its buffer) must sit inside the parent level's
    owned cells with 4 coarse cells of margin, so the prolongation stencil
    (coarse k-3..k+3 around a parent) reads only coarse blocks' own cells or
    their synchronised ghosts, and patches of a level must not touch."""
    for lev in range(1, len(self.levels)):
        for p in self.levels[lev]:
            _check(all(v % 2 == 0 for v in p.ext_lo + p.ext_hi), "refined patch boxes must be even")
            clo = [v // 2 for v in p.ext_lo]
            chi = [v // 2 for v in p.ext_hi]
            ok = False
            for q in self.levels[lev - 1]:
                if all(q.lo[d] + 4 <= clo[d] and chi[d] + 4 <= q.hi[d] for d in range(3)):
                    ok = True
            _check(ok, f"level {lev} patch {p.lo}-{p.hi} is not nested in level {lev - 1} with a 4-cell margin")
        pl = self.levels[lev]
        for a in range(len(pl)):
            for b in range(a + 1, len(pl)):
                _check(not all(pl[a].ext_lo[d] <= pl[b].ext_hi[d] and pl[b].ext_lo[d] <= pl[a].ext_hi[d]
                               for d in range(3)), f"level {lev} patches touch")


Hierarchy.check_nesting = _hierarchy_check
