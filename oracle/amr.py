"""CPU oracle of a Berger-Oliger evolution over a block hierarchy (test infrastructure only).

Follows, block by block and in the reference's order:
  bssn_class::RecursiveStep   bssn_class.C:2323-2414 (PSTR 0, RPS 1, trfls 0)
  bssn_class::Step            bssn_class.C:2981-3915 (per block substep via
                              oracle_bssn_substep, then Parallel::Sync)
  bssn_class::RestrictProlong bssn_class.C:5724-5903
  Parallel::prepare_inter_time_level Parallel.C:4329-4441 (average / average2)
with restrict3 / prolong3 from amr_oracle.c.  The hierarchy (patches, buffer
cells, blocks, ghost cells) is the plain description of
amss_b200.hierarchy.Hierarchy.  Parity unpinned (see oracle_common.h).
"""
import ctypes

import numpy as np

import oracle as O

_DP = ctypes.POINTER(ctypes.c_double)
_I3 = ctypes.c_int * 3


def _p(a):
    return a.ctypes.data_as(_DP)


def _ptrs(arr):
    return (_DP * arr.shape[0])(*[_p(arr[f]) for f in range(arr.shape[0])])


def _isect(alo, ahi, blo, bhi):
    lo = tuple(max(a, b) for a, b in zip(alo, blo))
    hi = tuple(min(a, b) for a, b in zip(ahi, bhi))
    return (lo, hi) if all(l < h for l, h in zip(lo, hi)) else None


class OracleHierarchy:
    def __init__(self, H, eps=0.1, chitiny=1e-5 - 1.0, symmetry=0, nf=24):
        """nf = 25: the Z4c evolution (Theta as the 25th field)."""
        self.H = H
        self.nf = nf
        self.eps = eps
        self.chitiny = chitiny
        self.symmetry = symmetry
        lib = O.lib()
        lib.oracle_evolve_substep.restype = ctypes.c_int
        self.blk = []
        for b in H.blocks:
            shape = (nf, b.ex[2], b.ex[1], b.ex[0])
            X, Y, Z = H.coords(b)
            p = H.levels[b.level][b.patch]
            self.blk.append(dict(
                U=[np.zeros(shape) for _ in range(3)], K=np.zeros(shape), A=np.zeros(shape), B=np.zeros(shape),
                X=X, Y=Y, Z=Z, pbbox=np.array(H.patch_bbox(p)), ex=(ctypes.c_int * 3)(*b.ex)))
        self.cur = [0] * len(H.levels)
        self.steps = [0] * len(H.levels)
        self.porg0 = None   # tracked punctures (set_punctures)

    # puncture tracking -------------------------------------------------------
    def set_punctures(self, positions):
        """bssn_class::Step with MAPBH 0 (bssn_class.C:3360-3390, :3730-3760,
        :3804-3812, :3890-3898): positions advanced with the finest level's
        substeps by rungekutta4_scalar (rungekutta4_rout.f90:6-47), their
        right-hand side minus the shift of the substep's input state
        (compute_Porg_rhs, bssn_class.C:6879-6932) on the finest level."""
        self.porg0 = [list(map(float, p)) for p in positions]
        self.porg = [list(p) for p in self.porg0]
        self.prhs = [[0.0] * 3 for _ in self.porg0]

    def _track(self, level, sub, arrays, dt):
        import interp as OI
        states = [None] * len(self.H.blocks)
        for bi in arrays:
            states[bi] = arrays[bi]
        patches = OI.hierarchy_patches(self.H, level, states)
        src = self.porg0 if sub == 0 else self.porg
        for n, pos in enumerate([list(p) for p in src]):
            vals, found = OI.interp_points(patches, [tuple(pos)], [18, 19, 20],
                                           [(-1, 1, 1), (1, -1, 1), (1, 1, -1)], self.symmetry)
            if not found[0]:
                raise ValueError("a puncture left the finest level")
            for v in range(3):
                r = -vals[0][v]
                f0 = self.porg0[n][v]
                if sub == 0:
                    self.prhs[n][v] = r
                    pn = f0 + 0.5 * dt * r
                elif sub == 1:
                    self.prhs[n][v] = self.prhs[n][v] + 2.0 * r
                    pn = f0 + 0.5 * dt * r
                elif sub == 2:
                    self.prhs[n][v] = self.prhs[n][v] + 2.0 * r
                    pn = f0 + dt * r
                else:
                    pn = f0 + (1.0 / 6.0) * dt * (r + self.prhs[n][v])
                if (self.symmetry > 0 and v == 2) or (self.symmetry == 2 and v < 2):
                    pn = abs(pn)
                self.porg[n][v] = pn
        if sub == 3:
            self.porg0 = [list(p) for p in self.porg]

    # state access ------------------------------------------------------------
    def state(self, bi):
        b = self.H.blocks[bi]
        return self.blk[bi]["U"][self.cur[b.level]]

    def set_state(self, bi, st):
        self.state(bi)[...] = st

    def _arr(self, bi, which):
        d = self.blk[bi]
        if which == "state":
            return self.state(bi)
        return d[which]

    @staticmethod
    def _view(b, arr, lo, hi):
        sl = tuple(slice(lo[d] - b.org[d], hi[d] - b.org[d]) for d in (2, 1, 0))
        return arr[(slice(None),) + sl]

    # Parallel::Sync ------------------------------------------------------------
    def sync(self, level, which):
        ids = [i for p in self.H.levels[level] for i in p.blocks]
        for d in ids:
            bd = self.H.blocks[d]
            alo, ahi = bd.org, tuple(bd.org[k] + bd.ex[k] for k in range(3))
            for s in ids:
                if s == d:
                    continue
                bs = self.H.blocks[s]
                r = _isect(alo, ahi, bs.own_lo, bs.own_hi)
                if r:
                    self._view(bd, self._arr(d, which), *r)[...] = self._view(bs, self._arr(s, which), *r)

    # bssn_class::Step ----------------------------------------------------------
    def level_step(self, level, dt):
        lib = O.lib()
        ids = [i for p in self.H.levels[level] for i in p.blocks]
        c = self.cur[level]
        err = 0
        finest = self.porg0 is not None and level == len(self.H.levels) - 1
        for sub in range(4):
            if finest:
                key = {0: None, 1: "A", 2: "B", 3: "A"}[sub]
                self._track(level, sub, {bi: (self.blk[bi]["U"][c] if key is None else self.blk[bi][key])
                                         for bi in ids}, dt)
            for bi in ids:
                d = self.blk[bi]
                u0 = d["U"][c]
                src = {0: u0, 1: d["A"], 2: d["B"], 3: d["A"]}[sub]
                out = {0: d["A"], 1: d["B"], 2: d["A"], 3: d["U"][(c + 1) % 3]}[sub]
                err |= lib.oracle_evolve_substep(d["ex"], _p(d["X"]), _p(d["Y"]), _p(d["Z"]), _p(d["pbbox"]),
                                                 _ptrs(u0), _ptrs(src), _ptrs(out), _ptrs(d["K"]), ctypes.c_int(sub),
                                                 ctypes.c_double(dt), ctypes.c_double(self.eps),
                                                 ctypes.c_double(self.chitiny), ctypes.c_int(self.symmetry),
                                                 ctypes.c_int(level), ctypes.c_int(self.nf))
            if sub < 3:
                self.sync(level, "A" if sub != 1 else "B")
        self.cur[level] = (c + 1) % 3
        self.steps[level] += 1
        self.sync(level, "state")
        return err

    # bssn_class::RestrictProlong ------------------------------------------------
    def restrict_prolong(self, level, same_time):
        lib = O.lib()
        H = self.H
        cl = level - 1
        cids = [i for p in H.levels[cl] for i in p.blocks]
        if not same_time:
            c = self.cur[cl]
            for bi in cids:
                d = self.blk[bi]
                f1, f2, f3 = d["U"][c], d["U"][(c + 2) % 3], d["U"][(c + 1) % 3]
                if self.steps[cl] >= 2:
                    lib.oracle_average2(ctypes.c_long(f1.size), _p(f1), _p(f2), _p(f3), _p(d["K"]))
                else:
                    d["K"][...] = 0.5 * (f1 + f2)
        ctarget = "state" if same_time else "K"
        for p in H.levels[level]:
            cphys_lo = tuple(v // 2 for v in p.lo)
            cphys_hi = tuple(v // 2 for v in p.hi)
            for cb in cids:
                bc = H.blocks[cb]
                r = _isect(cphys_lo, cphys_hi, bc.org, tuple(bc.org[k] + bc.ex[k] for k in range(3)))
                if not r:
                    continue
                for fb in p.blocks:
                    bf = H.blocks[fb]
                    rr = _isect(r[0], r[1], tuple(v // 2 for v in bf.own_lo), tuple(v // 2 for v in bf.own_hi))
                    if not rr:
                        continue
                    carr = self._arr(cb, ctarget)
                    farr = self.state(fb)
                    for f in range(self.nf):
                        lib.oracle_restrict3_box(_I3(*bc.ex), _I3(*bc.org), _p(carr[f]), _I3(*bf.ex), _I3(*bf.org),
                                                 _p(farr[f]), _I3(*rr[0]), _I3(*rr[1]))
        self.sync(cl, ctarget)
        for p in H.levels[level]:
            elo, ehi = p.ext_lo, p.ext_hi
            slabs = []
            for d in range(3):
                lo_a, hi_a = list(elo), list(ehi)
                lo_b, hi_b = list(elo), list(ehi)
                for q in range(d):
                    lo_a[q] = lo_b[q] = p.lo[q]
                    hi_a[q] = hi_b[q] = p.hi[q]
                hi_a[d] = p.lo[d]
                lo_b[d] = p.hi[d]
                slabs += [(tuple(lo_a), tuple(hi_a)), (tuple(lo_b), tuple(hi_b))]
            for fb in p.blocks:
                bf = H.blocks[fb]
                for slo, shi in slabs:
                    r = _isect(slo, shi, bf.org, tuple(bf.org[k] + bf.ex[k] for k in range(3)))
                    if not r:
                        continue
                    for cb in cids:
                        bc = H.blocks[cb]
                        rr = _isect(r[0], r[1], tuple(2 * v for v in bc.own_lo), tuple(2 * v for v in bc.own_hi))
                        if not rr:
                            continue
                        carr = self._arr(cb, ctarget)
                        farr = self.state(fb)
                        for f in range(self.nf):
                            lib.oracle_prolong3_box(_I3(*bc.ex), _I3(*bc.org), _p(carr[f]), _I3(*bf.ex),
                                                    _I3(*bf.org), _p(farr[f]), _I3(*rr[0]), _I3(*rr[1]))
        self.sync(level, "state")

    # bssn_class::RecursiveStep ---------------------------------------------------
    def recursive_step(self, level, dt0):
        iters = 1 if level == 0 else 2
        dt = dt0 / 2 ** level
        err = 0
        for i in range(iters):
            yn = i == iters - 1
            err |= self.level_step(level, dt)
            if level < len(self.H.levels) - 1:
                err |= self.recursive_step(level + 1, dt0)
            if level > 0:
                self.restrict_prolong(level, yn)
        return err

    def coarse_step(self, dt0):
        return self.recursive_step(0, dt0)


    # cgh::recompose_cgh_Onelevel + Parallel::fill_level_data -----------------
    def regrid_fill(self, old, level, back):
        """Fill `level` of this hierarchy (the new boxes), time level `back`
        (0: current, 1: one level step before), from the hierarchy `old` it
        replaces (Parallel.C fill_level_data): cells of this level's arrays
        that an old block owns are copied; cells outside every old patch
        (buffers included) are prolonged (prolong3) from the old parent level,
        in time too for back = 1 (average2 of the parent's three levels, the
        mean of two before its second step).  The level's clock is copied."""
        lib = O.lib()
        H, Ho = self.H, old.H
        self.cur[level] = old.cur[level]
        self.steps[level] = old.steps[level]
        slot = (self.cur[level] + 3 - back) % 3
        oslot = (old.cur[level] + 3 - back) % 3
        new_ids = [i for p in H.levels[level] for i in p.blocks]
        old_ids = [i for p in Ho.levels[level] for i in p.blocks]
        for d in new_ids:
            bd = H.blocks[d]
            alo, ahi = bd.org, tuple(bd.org[k] + bd.ex[k] for k in range(3))
            for s_ in old_ids:
                bs = Ho.blocks[s_]
                r = _isect(alo, ahi, bs.own_lo, bs.own_hi)
                if r:
                    self._view(bd, self.blk[d]["U"][slot], *r)[...] = old._view(bs, old.blk[s_]["U"][oslot], *r)
        if level == 0:
            return
        # the parent's source values: current state, or interpolated in time
        cl = level - 1
        par_ids = [i for p in Ho.levels[cl] for i in p.blocks]
        src = {}
        for cb in par_ids:
            d_ = old.blk[cb]
            c = old.cur[cl]
            if back == 0:
                src[cb] = d_["U"][c]
            else:
                f1, f2, f3 = d_["U"][c], d_["U"][(c + 2) % 3], d_["U"][(c + 1) % 3]
                if old.steps[cl] >= 2:
                    t = np.empty_like(f1)
                    lib.oracle_average2(ctypes.c_long(f1.size), _p(f1), _p(f2), _p(f3), _p(t))
                else:
                    t = 0.5 * (f1 + f2)
                src[cb] = t
        for d in new_ids:
            bd = H.blocks[d]
            pieces = [(bd.org, tuple(bd.org[k] + bd.ex[k] for k in range(3)))]
            for p in Ho.levels[level]:
                nxt = []
                for lo, hi in pieces:
                    nxt += _subtract(lo, hi, p.ext_lo, p.ext_hi)
                pieces = nxt
            farr = self.blk[d]["U"][slot]
            for lo, hi in pieces:
                for cb in par_ids:
                    bc = Ho.blocks[cb]
                    rr = _isect(lo, hi, tuple(2 * v for v in bc.own_lo), tuple(2 * v for v in bc.own_hi))
                    if not rr:
                        continue
                    for f in range(self.nf):
                        lib.oracle_prolong3_box(_I3(*bc.ex), _I3(*bc.org), _p(src[cb][f]), _I3(*bd.ex),
                                                _I3(*bd.org), _p(farr[f]), _I3(*rr[0]), _I3(*rr[1]))


def _subtract(alo, ahi, blo, bhi):
    """The box [alo, ahi) less [blo, bhi), as disjoint boxes."""
    r = _isect(alo, ahi, blo, bhi)
    if not r:
        return [(tuple(alo), tuple(ahi))]
    out = []
    lo, hi = list(alo), list(ahi)
    for d in range(3):
        if lo[d] < r[0][d]:
            h2 = list(hi)
            h2[d] = r[0][d]
            out.append((tuple(lo), tuple(h2)))
            lo[d] = r[0][d]
        if r[1][d] < hi[d]:
            l2 = list(lo)
            l2[d] = r[1][d]
            out.append((tuple(l2), tuple(hi)))
            hi[d] = r[1][d]
    return out


def regrid_onelevel(lev, boxes, handles, porgls, porg0, x0, h0, symmetry=0):
    """cgh::Regrid_Onelevel's box move (cgh.C:1340-1470) for one level:
    boxes[grd] = [lo, hi] in the level's global cells (moved in place),
    handles[grd] their centres (moved in place), porgls[bh] the punctures'
    positions at the level's last regrid, porg0[bh] the current ones.
    Returns (moved, new porgls)."""
    do_every = 2
    nbh = len(porg0)
    dX = h0 * 0.5 ** lev
    tmp = [list(p) for p in porgls]
    tot_flag = False
    for grd in range(len(boxes)):
        bhi = 0
        while bhi < nbh:
            if (abs(porgls[bhi][0] - handles[grd][0]) < 2 * do_every * dX and
                    abs(porgls[bhi][1] - handles[grd][1]) < 2 * do_every * dX and
                    abs(porgls[bhi][2] - handles[grd][2]) < 2 * do_every * dX):
                break
            bhi += 1
        if bhi == nbh:
            blo = [x0 + boxes[grd][0][d] * dX for d in range(3)]
            if abs(blo[0]) < dX / 2 and abs(blo[1]) < dX / 2 and abs(blo[2]) < dX / 2:
                break
            if nbh == 1:
                bhi = 0
            else:
                raise ValueError("no black hole matches the box")
        for d in range(3):
            rr = (porg0[bhi][d] - handles[grd][d]) / dX
            flag = int(rr + 0.5) if rr > 0 else int(rr - 0.5)       # Python int() truncates like C
            flag = int(flag / do_every) * do_every
            shift = flag * dX
            if abs(shift) > dX / 2:
                tot_flag = True
                boxes[grd][0][d] += flag
                boxes[grd][1][d] += flag
                handles[grd][d] += shift
                tmp[bhi][d] = porg0[bhi][d]
    return tot_flag, (tmp if tot_flag else porgls)


def grid_noise(level, field, gi, gj, gk, seed):
    """Uniform noise in [-1, 1) as a function of (seed, level, field, global
    cell index) only, so every copy of a cell (owner, ghost, buffer) agrees.
    splitmix64 finaliser over the packed key (64-bit wrap-around intended)."""
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)
               ^ (np.uint64(level) << np.uint64(56)) ^ (np.uint64(field) << np.uint64(48))
               ^ ((gk.astype(np.uint64) & np.uint64(0xFFFF)) << np.uint64(32))
               ^ ((gj.astype(np.uint64) & np.uint64(0xFFFF)) << np.uint64(16))
               ^ (gi.astype(np.uint64) & np.uint64(0xFFFF)))
        z = key + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 / 2.0 ** 53) - 1.0


def initial_state(H, masses, positions, noise=0.0, seed=1, nf=24):
    """Brill-Lindquist data on every block (get_lousto_nbhs), plus uniform noise
    of amplitude `noise` that depends only on the global cell (grid_noise).
    nf = 25 appends the Z4c Theta field (zero, plus the same kind of noise)."""
    out = []
    with np.errstate(over="ignore"):
        for b in H.blocks:
            X, Y, Z = H.coords(b)
            st = O.brill_lindquist(X, Y, Z, masses, positions)
            if nf == 25:
                st = np.concatenate([st, np.zeros((1,) + st.shape[1:])])
            if noise > 0:
                gk, gj, gi = np.meshgrid(np.arange(b.ex[2]) + b.org[2], np.arange(b.ex[1]) + b.org[1],
                                         np.arange(b.ex[0]) + b.org[0], indexing="ij")
                for f in range(nf):
                    st[f] += noise * grid_noise(b.level, f, gi, gj, gk, seed)
            out.append(st)
    return out
