"""CPU oracle of point interpolation on a level (test infrastructure only).

Restates, in plain Python floats (IEEE double, no fused multiply-add):
  Parallel::PatList_Interp_Points  Parallel.C:5614-5667  (first patch whose
                                   box less its buffer holds the point)
  Patch::Interp_Points             MPatch.C:339-500 (Cell: first block whose
                                   box less its ghosts, or less the buffer on a
                                   patch side, holds the point to DH/2)
  global_interp                    fmisc.f90:712-794 (ORDN = 2 ghost_width = 6)
  decide3d                         fmisc.f90:798-874 (mirrored cells times SoA)
  polin3 / polint                  fmisc.f90:1121-1260 (Neville, z then y then x)
The hierarchy is amss_b200.hierarchy.Hierarchy; blocks added by bbox are given
as (bbox, patch_bbox) pairs.  Parity unpinned (see oracle_common.h): checked
against polynomial exactness in the tests.
"""
GHOST = 3
ORDN = 2 * GHOST


def polint(xa, ya, x):
    """fmisc.f90:1121-1179."""
    n = len(xa)
    c = list(ya)
    d = list(ya)
    ho = [xa[i] - x for i in range(n)]
    ns = 1
    dif = abs(x - xa[0])
    for m in range(1, n + 1):
        dift = abs(x - xa[m - 1])
        if dift < dif:
            ns = m
            dif = dift
    y = ya[ns - 1]
    ns -= 1
    for m in range(1, n):
        den = [ho[i] - ho[i + m] for i in range(n - m)]
        if any(v == 0.0 for v in den):
            raise ZeroDivisionError("failure in polint")
        den = [(c[i + 1] - d[i]) / den[i] for i in range(n - m)]
        for i in range(n - m):
            d[i] = ho[i + m] * den[i]
        for i in range(n - m):
            c[i] = ho[i] * den[i]
        if 2 * ns < n - m:
            dy = c[ns]          # c(ns+1), 1-based
        else:
            dy = d[ns - 1]      # d(ns)
            ns -= 1
        y = y + dy
    return y


def polin3(ya, x1, x2, x3):
    """fmisc.f90:1221-1260; ya[i][j][k] with 0-based i, j, k < ORDN."""
    xa = [float(j) for j in range(ORDN)]
    ym = []
    for i in range(ORDN):
        yat = [polint(xa, ya[i][j], x3) for j in range(ORDN)]
        ym.append(polint(xa, yat, x2))
    return polint(xa, ym, x1)


def global_interp(f, X, Y, Z, x1, y1, z1, soa, symmetry):
    """fmisc.f90:712-794.  f: one field (ez, ey, ex) numpy array; soa: the
    field's parities (x, y, z)."""
    ex = (len(X), len(Y), len(Z))
    co = (X, Y, Z)
    p = (x1, y1, z1)
    dd = [co[m][1] - co[m][0] for m in range(3)]
    cxI = [int((p[m] - co[m][0]) / dd[m] + 0.4) + 1 for m in range(3)]
    cxB = [cxI[m] - ORDN // 2 + 1 for m in range(3)]
    cxT = [cxB[m] + ORDN - 1 for m in range(3)]
    cmin = [1, 1, 1]
    cmax = list(ex)
    if symmetry == 2 and abs(X[0]) < dd[0]:
        cmin[0] = -ORDN // 2 + 1
    if symmetry == 2 and abs(Y[0]) < dd[1]:
        cmin[1] = -ORDN // 2 + 1
    if symmetry != 0 and abs(Z[0]) < dd[2]:
        cmin[2] = -ORDN // 2 + 1
    for m in range(3):
        if cxB[m] < cmin[m]:
            cxB[m] = cmin[m]
            cxT[m] = cxB[m] + ORDN - 1
        if cxT[m] > cmax[m]:
            cxT[m] = cmax[m]
            cxB[m] = cxT[m] + 1 - ORDN
    cx = []
    for m in range(3):
        if cxB[m] > 0:
            cx.append((p[m] - co[m][cxB[m] - 1]) / dd[m])
        else:
            cx.append((p[m] + co[m][1 - cxB[m] - 1]) / dd[m])
    # decide3d: the cube, mirrored (times the parities) where an index is <= 0
    for m in range(3):
        if cxT[m] > ex[m] or (cxB[m] <= 0 and 1 - cxB[m] > ex[m]):
            raise ValueError("error in decide3d")
    ya = [[[0.0] * ORDN for _ in range(ORDN)] for _ in range(ORDN)]
    for a in range(ORDN):
        i = cxB[0] + a
        for b in range(ORDN):
            j = cxB[1] + b
            for c in range(ORDN):
                k = cxB[2] + c
                v = float(f[(k if k > 0 else 1 - k) - 1, (j if j > 0 else 1 - j) - 1, (i if i > 0 else 1 - i) - 1])
                if i <= 0:
                    v = v * soa[0]
                if j <= 0:
                    v = v * soa[1]
                if k <= 0:
                    v = v * soa[2]
                ya[a][b][c] = v
    return polin3(ya, cx[0], cx[1], cx[2])


def _in_patch(pt, pbb, buffer, shape):
    for m in range(3):
        h = (pbb[3 + m] - pbb[m]) / shape[m]
        if pt[m] < pbb[m] + buffer * h or pt[m] > pbb[3 + m] - buffer * h:
            return False
    return True


def _in_block(pt, bb, pbb, buffer, shape):
    for m in range(3):
        h = (pbb[3 + m] - pbb[m]) / shape[m]
        lo = bb[m] + buffer * h if abs(bb[m] - pbb[m]) < h / 2 else bb[m] + GHOST * h
        hi = bb[3 + m] - buffer * h if abs(bb[3 + m] - pbb[3 + m]) < h / 2 else bb[3 + m] - GHOST * h
        if pt[m] - lo < -h / 2 or pt[m] - hi > h / 2:
            return False
    return True


def interp_points(patches, points, fields, soas, symmetry=0):
    """patches: list of (patch_bbox, shape, buffer, [(bbox, X, Y, Z, state), ...])
    in the level's order; returns (values [npts][nvar], found [npts]).  A point
    in a patch but in none of its blocks raises, as the reference aborts."""
    vals, found = [], []
    for pt in points:
        row = [0.0] * len(fields)
        ok = False
        for pbb, shape, buffer, blocks in patches:
            if not _in_patch(pt, pbb, buffer, shape):
                continue
            for bb, X, Y, Z, st in blocks:
                if _in_block(pt, bb, pbb, buffer, shape):
                    row = [global_interp(st[f], X, Y, Z, pt[0], pt[1], pt[2], soas[v], symmetry)
                           for v, f in enumerate(fields)]
                    ok = True
                    break
            if not ok:
                raise ValueError(f"Patch::Interp_Points fails to find point {pt}")
            break
        vals.append(row)
        found.append(ok)
    return vals, found


def hierarchy_patches(H, level, states):
    """interp_points' patch list for one level of a Hierarchy."""
    out = []
    for p in H.levels[level]:
        pbb = H.patch_bbox(p)
        shape = [p.ext_hi[m] - p.ext_lo[m] for m in range(3)]
        blocks = []
        for bi in p.blocks:
            b = H.blocks[bi]
            X, Y, Z = H.coords(b)
            blocks.append((H.bbox(b), X, Y, Z, states[bi]))
        out.append((pbb, shape, p.buffer, blocks))
    return out
