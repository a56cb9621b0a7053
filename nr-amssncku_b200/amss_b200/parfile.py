"""The reference's parameter file (AMSS-NCKU.input) as an engine configuration.

The reference's Python front end writes `Group::key = value` lines
(setup.py:388-450 ABE::, numerical_grid.py:558-669 cgh::,
renew_puncture_parameter.py:103-127 BSSN::) that the C++ driver reads with
misc::parse_parts (misc.C:71-112, and the three-index form for
cgh::shape[l][g][d] / cgh::bbox[l][g][d]).  This module reads the same file
by the same rules and turns it into what the batched engine needs:

* the grid hierarchy of cgh::levels / grids / shape / bbox (cgh.C:1018-1080):
  level 0's box and cell count fix the origin and h0; every box of a finer
  level is aligned to that level's cells as Parallel::aligncheck
  (Parallel.C:5724-5760) does and must have the cell count it is given; the
  boxes of a level merge as amss_b200.hierarchy.merge_boxes describes, and
  each patch is split into seeded uneven blocks;
* ABE::Symmetry, ABE::Courant (dT = Courant * min dx, bssn_class.C:717-721),
  the dissipation (ABE::big dissipation below cgh::moving levels start from,
  ABE::small dissipation from there, bssn_class.C:3032-3034; the engine takes
  one eps, so the two must agree), BSSN::chitiny, and the punctures
  BSSN::Mass / Porg / Pmom / Spin for ABE::ID Type -1 (Lousto's approximate
  data, get_lousto_nbhs_).

What the engine does not implement is refused with AmssError rather than
silently dropped: shells, time refinement starting above level 0, unequal
dissipation per level kind, non-cubic cells, initial data other than Lousto's.
"""
from dataclasses import dataclass, field

import numpy as np

from ._lib import AmssError
from .hierarchy import from_boxes


class ParError(AmssError):
    pass


def _ltrim(s):
    return s.lstrip(" \t\r\n")


def _rtrim(s):
    return s.rstrip(" \t\r\n")


def parse_line(line):
    """misc::parse_parts (misc.C:71-112, three-index form :136-196): returns
    None for a blank or comment line, else (group, key, value, (i1, i2, i3));
    a line without both '::' and '=' is an error, as the driver aborts on it."""
    s = line.split("#", 1)[0]
    if not _rtrim(s):
        return None
    p1, p2 = s.find("::"), s.find("=")
    if p1 < 0 or p2 < 0:
        raise ParError(f"malformed parameter line: {line.rstrip()!r}")
    grp = _ltrim(s[:p1])
    key = _rtrim(s[p1 + 2:p2])
    val = s[p2 + 1:].strip(" \t\r\n")
    q1, q2 = val.find('"'), val.rfind('"')
    if q1 >= 0:
        val = val[1:q2]
    idx = [0, 0, 0]
    rest = ""
    b1, b2 = key.find("["), key.find("]")
    if b1 >= 0:
        rest = key[b2 + 1:]
        idx[0] = _atoi(key[b1 + 1:b2])
        key = key[:b1]
    for n in (1, 2):
        b1, b2 = rest.find("["), rest.find("]")
        if b1 < 0:
            break
        idx[n] = _atoi(rest[b1 + 1:b2])
        rest = rest[b2 + 1:]
    return grp, key, val, tuple(idx)


def _atoi(s):
    s = s.strip()
    n = 0
    while n < len(s) and (s[n].isdigit() or (n == 0 and s[n] in "+-")):
        n += 1
    try:
        return int(s[:n])
    except ValueError:
        return 0


class ParFile:
    """All entries of a parameter file; a later line overrides an earlier one
    with the same group, key and indices (the driver's reads assign in file
    order)."""

    def __init__(self, text):
        self.entries = {}
        for ln in text.splitlines():
            e = parse_line(ln)
            if e is not None:
                grp, key, val, idx = e
                self.entries[(grp, key, idx)] = val

    @classmethod
    def read(cls, path):
        with open(path) as f:
            return cls(f.read())

    def has(self, grp, key, *idx):
        return (grp, key, tuple(idx) + (0,) * (3 - len(idx))) in self.entries

    def get(self, grp, key, *idx, default=None, conv=str):
        k = (grp, key, tuple(idx) + (0,) * (3 - len(idx)))
        if k not in self.entries:
            if default is None:
                raise ParError(f"parameter {grp}::{key}{''.join(f'[{i}]' for i in idx)} is missing")
            return default
        v = self.entries[k]
        if conv is int:
            return _atoi(v)
        if conv is float:
            return float(v.replace("d", "e").replace("D", "e"))
        return v


@dataclass
class RunConfig:
    """Everything the engine takes from a parameter file."""
    hierarchy: object
    symmetry: int
    eps: float
    chitiny: float            # BSSN::chitiny as written (the engine shifts it by -1)
    courant: float
    dt0: float                # coarse time step, Courant * min dx of level 0
    masses: list = field(default_factory=list)
    positions: list = field(default_factory=list)
    momenta: list = field(default_factory=list)
    spins: list = field(default_factory=list)

    def engine(self, precision="fp64", formulation="bssn", **kw):
        """An amss_b200.Engine over the hierarchy with these parameters."""
        from .engine import Engine
        return Engine.from_hierarchy(self.hierarchy, precision=precision, symmetry=self.symmetry, eps=self.eps,
                                     chitiny=self.chitiny, formulation=formulation, **kw)

    def initial_state(self, noise=0.0, seed=1, nf=24):
        """Lousto's puncture data on every block (get_lousto_nbhs_ on the GPU)."""
        from . import initial
        if any(np.any(np.asarray(p) != 0) for p in self.momenta + self.spins):
            raise ParError("initial data with puncture momenta or spins: only the Brill-Lindquist case is wired up")
        return initial.initial_state(self.hierarchy, self.masses, self.positions, noise=noise, seed=seed, nf=nf)


def _hierarchy(par, seed, block_min, block_max):
    levels = par.get("cgh", "levels", conv=int)
    if levels < 1:
        raise ParError("cgh::levels must be >= 1")
    grids = [par.get("cgh", "grids", lv, conv=int) for lv in range(levels)]
    if grids[0] != 1:
        raise ParError("level 0 must be one box (shell-patch grids are not supported)")

    def box(lv, g):
        bb = [par.get("cgh", "bbox", lv, g, d, conv=float) for d in range(6)]
        sh = [par.get("cgh", "shape", lv, g, d, conv=int) for d in range(3)]
        return bb, sh

    bb0, sh0 = box(0, 0)
    dh0 = [(bb0[3 + d] - bb0[d]) / sh0[d] for d in range(3)]   # Cell: (bbox_hi - bbox_lo) / shape
    if max(dh0) - min(dh0) > 1e-12 * max(dh0) or max(bb0[:3]) - min(bb0[:3]) > 1e-12 * max(1.0, abs(bb0[0])):
        raise ParError("level 0 must have cubic cells and one origin on every axis")
    x0, h0 = bb0[0], dh0[0]
    out = []
    for lv in range(1, levels):
        hl = h0 * 0.5 ** lv
        boxes = []
        for g in range(grids[lv]):
            bb, sh = box(lv, g)
            lo, hi = [], []
            for d in range(3):
                # Parallel::aligncheck: snap the box onto the level's cells, then
                # its cell count must be the one given
                blo = bb0[d] + int((bb[d] - bb0[d]) / hl + 0.4) * hl
                bhi = bb0[3 + d] - int((bb0[3 + d] - bb[3 + d]) / hl + 0.4) * hl
                nn = int((bhi - blo) / hl + 0.4)
                if nn != sh[d]:
                    raise ParError(f"cgh box {lv}/{g}: aligned extent has {nn} cells along axis {d}, shape says {sh[d]}")
                i0 = int(round((blo - x0) / hl))
                lo.append(i0)
                hi.append(i0 + nn)
            if any(v % 2 for v in lo + hi):
                raise ParError(f"cgh box {lv}/{g} does not start and end on parent cells")
            boxes.append([lo, hi])
        out.append(boxes)
    return from_boxes(x0, h0, tuple(sh0), out, seed=seed, block_min=block_min, block_max=block_max)


def load(path_or_text, seed=1, block_min=24, block_max=80):
    """RunConfig of a parameter file (a path, or the file's text if it holds
    a newline).  Blocks: seeded uneven splits of block_min..block_max cells."""
    par = ParFile(path_or_text) if "\n" in path_or_text else ParFile.read(path_or_text)
    sym = par.get("ABE", "Symmetry", conv=int)
    if sym not in (0, 1, 2):
        raise ParError("ABE::Symmetry must be 0, 1 or 2")
    movls = par.get("cgh", "moving levels start from", conv=int)
    levels = par.get("cgh", "levels", conv=int)
    small = par.get("ABE", "small dissipation", conv=float)
    big = par.get("ABE", "big dissipation", conv=float)
    if movls < levels and movls > 0 and small != big:
        raise ParError("different dissipation on fixed and moving levels is not supported (one eps per engine)")
    eps = small if movls == 0 else (big if movls >= levels else small)
    trfls = par.get("BSSN", "time refinement start from level", conv=int, default="0")
    if trfls != 0:
        raise ParError("time refinement must start from level 0 (BSSN::time refinement start from level = 0)")
    idt = par.get("ABE", "ID Type", conv=int, default="-1")
    if idt != -1:
        raise ParError(f"ABE::ID Type {idt}: only Lousto's analytic puncture data (-1) is supported")
    H = _hierarchy(par, seed, block_min, block_max)
    courant = par.get("ABE", "Courant", conv=float)
    nbh = par.get("BSSN", "BH_num", conv=int, default="0")
    f = lambda k, i: par.get("BSSN", k, i, conv=float, default="0")   # noqa: E731
    return RunConfig(
        hierarchy=H, symmetry=sym, eps=eps, chitiny=par.get("BSSN", "chitiny", conv=float, default="1e-5"),
        courant=courant, dt0=courant * H.h0,
        masses=[f("Mass", i) for i in range(nbh)],
        positions=[[f("Porgx", i), f("Porgy", i), f("Porgz", i)] for i in range(nbh)],
        momenta=[[f("Pmomx", i), f("Pmomy", i), f("Pmomz", i)] for i in range(nbh)],
        spins=[[f("Spinx", i), f("Spiny", i), f("Spinz", i)] for i in range(nbh)])
