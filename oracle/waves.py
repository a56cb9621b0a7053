"""CPU oracle of the wave extraction (test infrastructure only).

Restates:
  bssn_class::Compute_Psi4   bssn_class.C:6210-6298 (getnp4 on every block of
                             the level, then Parallel::Sync of Rpsi4 / Ipsi4)
  getnp4                     getnp4.f90:12-452 (psi4_oracle.c)
  surface_integral::surface_integral  surface_integral.C:39-181 (GaussInt:
                             Gauss-Legendre in cos(theta), midpoint in phi,
                             N_theta = 2N, N_phi = 4N, halved per symmetry)
  surface_integral::surf_Wave surface_integral.C:197-377 (spin-weight -2
                             modes l = 2..maxl, m = -l..l)
  misc::gaulegf, inversearray, Wigner_d_function, fact  misc.C:226-308
The Christoffel symbols and Ricci tensor getnp4 takes are compute_rhs_bssn's
(oracle.compute_rhs_bssn) of the same state.  Parity unpinned (oracle_common.h).
"""
import ctypes
import math

import numpy as np

import interp as OI
import oracle as O

PI = math.pi
RPSI4_SOA = (1.0, 1.0, 1.0)      # bssn_class.C:347-348
IPSI4_SOA = (-1.0, -1.0, -1.0)


def getnp4(X, Y, Z, state, gamma, ricci, symmetry=0):
    """getnp4.f90:12-452 on one block: (Rpsi4, Ipsi4)."""
    L = O.lib()
    shp = state.shape[1:]
    ex = O._ex(shp)
    st = np.ascontiguousarray(state, dtype=np.float64)
    g = np.ascontiguousarray(gamma, dtype=np.float64)
    r = np.ascontiguousarray(ricci, dtype=np.float64)
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    rp = np.zeros(shp)
    ip = np.zeros(shp)
    G = (O._DP * 18)(*[O._p(g[a]) for a in range(18)])
    R = (O._DP * 6)(*[O._p(r[a]) for a in range(6)])
    # state order: chi trK gxx gxy gxz gyy gyz gzz Axx Axy Axz Ayy Ayz Azz
    L.oracle_getnp4(ex, O._p(X), O._p(Y), O._p(Z), *[O._p(st[f]) for f in range(14)], G, R, O._p(rp), O._p(ip),
                    ctypes.c_int(symmetry))
    return rp, ip


def psi4_level(H, level, states, symmetry=0, eps=0.1):
    """Compute_Psi4 of one level: getnp4 on every block (Christoffel and Ricci
    from compute_rhs_bssn of the same state), then the same-level sync (each
    block's cells that another block owns copied from it).  Returns per block
    an array (2, ez, ey, ex): Rpsi4, Ipsi4."""
    ids = [bi for p in H.levels[level] for bi in p.blocks]
    out = {}
    for bi in ids:
        b = H.blocks[bi]
        X, Y, Z = H.coords(b)
        _, _, gam, ric, _ = O.compute_rhs_bssn(X, Y, Z, states[bi], symmetry=symmetry, lev=level, eps=eps)
        rp, ip = getnp4(X, Y, Z, states[bi], gam, ric, symmetry)
        out[bi] = np.stack([rp, ip])
    for d in ids:
        bd = H.blocks[d]
        alo, ahi = bd.org, tuple(bd.org[k] + bd.ex[k] for k in range(3))
        for s in ids:
            if s == d:
                continue
            bs = H.blocks[s]
            lo = tuple(max(alo[k], bs.own_lo[k]) for k in range(3))
            hi = tuple(min(ahi[k], bs.own_hi[k]) for k in range(3))
            if any(lo[k] >= hi[k] for k in range(3)):
                continue
            dsl = tuple(slice(lo[k] - bd.org[k], hi[k] - bd.org[k]) for k in (2, 1, 0))
            ssl = tuple(slice(lo[k] - bs.org[k], hi[k] - bs.org[k]) for k in (2, 1, 0))
            out[d][(slice(None),) + dsl] = out[s][(slice(None),) + ssl]
    return out


def fact(n):
    """misc.C:298-308."""
    return 1.0 if n == 0 else n * fact(n - 1)


def wigner_d(l, m, s, costheta):
    """misc.C:271-297: d^l_{m,s}(theta) by its explicit sum, even terms then
    odd terms as the reference adds them."""
    C1, C2 = max(0, m - s), min(l + m, l - s)
    vv = 0.0
    sinht = math.sqrt((1 - costheta) / 2.0)
    cosht = math.sqrt((1 + costheta) / 2.0)

    def term(t):
        return math.pow(cosht, 2 * l + m - s - 2 * t) * math.pow(sinht, 2 * t + s - m) / (
            fact(l + m - t) * fact(l - s - t) * fact(t) * fact(t + s - m))

    even = C1 % 2 == 0
    for t in range(C1, C2 + 1, 2):
        vv = vv + term(t) if even else vv - term(t)
    for t in range(C1 + 1, C2 + 1, 2):
        vv = vv - term(t) if even else vv + term(t)
    return vv * math.sqrt(fact(l + m) * fact(l - m) * fact(l + s) * fact(l - s))


def gaulegf(x1, x2, n):
    """misc.C:226-257 (Newton on P_n from cos(pi (i + 0.75)/(n + 0.5)))."""
    x = [0.0] * n
    w = [0.0] * n
    eps = 1.2e-16
    m = (n + 1) // 2
    xm = 0.5 * (x2 + x1)
    xl = 0.5 * (x2 - x1)
    for i in range(m):
        z = math.cos(PI * (i + 0.75) / (n + 0.5))
        while True:
            p1, p2 = 1.0, 0.0
            for j in range(n):
                p3 = p2
                p2 = p1
                p1 = ((2 * j + 1) * z * p2 - j * p3) / (j + 1)
            pp = n * (z * p1 - p2) / (z * z - 1.0)
            z1 = z
            z = z1 - p1 / pp
            if abs(z - z1) <= eps:
                break
        x[i] = xm - xl * z
        x[n - 1 - i] = xm + xl * z
        w[i] = 2.0 * xl / ((1.0 - z * z) * pp * pp)
        w[n - 1 - i] = w[i]
    return x, w


def sphere(nquarter, symmetry):
    """surface_integral.C:39-181 with GaussInt: (costheta nodes, weights,
    N_theta, N_phi, dphi, points (n_tot, 3) on the unit sphere)."""
    n_phi, n_theta = 4 * nquarter, 2 * nquarter
    ct, wt = gaulegf(-1.0, 1.0, n_theta)
    ct, wt = ct[::-1], wt[::-1]   # misc::inversearray: the upper half first
    if symmetry == 2:
        n_phi, n_theta = n_phi // 4, n_theta // 2
        dphi = PI / (2.0 * n_phi)
    elif symmetry == 1:
        n_theta = n_theta // 2
        dphi = 2.0 * PI / n_phi
    else:
        dphi = 2.0 * PI / n_phi
    pts = []
    for i in range(n_theta):
        c = ct[i]
        s = math.sqrt(1.0 - c * c)
        for j in range(n_phi):
            ph = (j + 0.5) * dphi
            pts.append((s * math.cos(ph), s * math.sin(ph), c))
    return ct, wt, n_theta, n_phi, dphi, pts


def surf_wave(rex, values, nquarter, symmetry, maxl, spinw=2):
    """surface_integral.C:197-377 (GaussInt) given the interpolated (Rpsi4,
    Ipsi4) at the sphere's points (n_tot x 2, sphere() order): returns (RP, IP)
    of the modes l = spinw..maxl, m = -l..l."""
    ct, wt, n_theta, n_phi, dphi, _ = sphere(nquarter, symmetry)
    nn = sum(2 * l + 1 for l in range(spinw, maxl + 1))
    rp = [0.0] * nn
    ip = [0.0] * nn
    lpsy = {0: 1, 1: 2, 2: 8}[symmetry]
    sR, sI = RPSI4_SOA, IPSI4_SOA
    for n in range(n_theta * n_phi):
        i = n // n_phi
        j = n - i * n_phi
        c = 0
        for pl in range(spinw, maxl + 1):
            for pm in range(-pl, pl + 1):
                for lp in range(lpsy):
                    R, I = values[n][0], values[n][1]
                    a = (j + 0.5) * dphi            # cos(pm * (j + 0.5) * dphi) associates as (pm * (j + 0.5)) * dphi
                    pa = pm * (j + 0.5) * dphi
                    if lp == 0:
                        cth, cm, sm, r, im = ct[i], math.cos(pa), math.sin(pa), R, I
                    elif lp == 1:
                        cth, cm, sm, r, im = -ct[i], math.cos(pa), math.sin(pa), sR[2] * R, sI[2] * I
                    elif lp == 2:
                        cth, cm, sm, r, im = ct[i], math.cos(pa), -math.sin(pa), sR[1] * R, sI[1] * I
                    elif lp == 3:
                        cth, cm, sm = -ct[i], math.cos(pa), -math.sin(pa)
                        r, im = sR[2] * sR[1] * R, sI[2] * sI[1] * I
                    elif lp == 4:
                        cth, cm, sm, r, im = ct[i], math.cos(pm * (PI - a)), math.sin(pm * (PI - a)), sR[0] * R, sI[0] * I
                    elif lp == 5:
                        cth, cm, sm = -ct[i], math.cos(pm * (PI - a)), math.sin(pm * (PI - a))
                        r, im = sR[2] * sR[0] * R, sI[2] * sI[0] * I
                    elif lp == 6:
                        cth, cm, sm = ct[i], math.cos(pm * (PI + a)), math.sin(pm * (PI + a))
                        r, im = sR[1] * sR[0] * R, sI[1] * sI[0] * I
                    else:
                        cth, cm, sm = -ct[i], math.cos(pm * (PI + a)), math.sin(pm * (PI + a))
                        r, im = sR[2] * sR[1] * sR[0] * R, sI[2] * sI[1] * sI[0] * I
                    th = math.sqrt((2 * pl + 1.0) / 4.0 / PI) * wigner_d(pl, pm, spinw, cth)
                    rp[c] = rp[c] + th * (r * cm + im * sm) * wt[i]
                    ip[c] = ip[c] + th * (im * cm - r * sm) * wt[i]
                c += 1
    return [v * rex * dphi for v in rp], [v * rex * dphi for v in ip]


def extract(H, level, psi4, rex, nquarter, maxl, symmetry=0):
    """Compute_Psi4's arrays interpolated on the sphere of radius rex
    (Patch::Interp_Points of the level) and decomposed by surf_Wave."""
    _, _, _, _, _, pts = sphere(nquarter, symmetry)
    P = OI.hierarchy_patches(H, level, psi4)
    vals, found = OI.interp_points(P, [(rex * a, rex * b, rex * c) for a, b, c in pts], [0, 1],
                                   [RPSI4_SOA, IPSI4_SOA], symmetry)
    if not all(found):
        raise ValueError("a sphere point lies outside the level")
    return surf_wave(rex, vals, nquarter, symmetry, maxl)


def admmass(X, Y, Z, state, symmetry=0):
    """admmass_bssn (fadmquantites_bssn.f90:5-65) on one block: (3, ez, ey, ex)."""
    L = O.lib()
    shp = state.shape[1:]
    st = np.ascontiguousarray(state, dtype=np.float64)
    out = np.zeros((3,) + shp)
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    f = [0, 2, 3, 4, 5, 6, 7, 14, 15, 16]   # chi, the metric, Gam^i
    L.oracle_admmass_bssn(O._ex(shp), O._p(X), O._p(Y), O._p(Z), *[O._p(st[k]) for k in f],
                          O._p(out[0]), O._p(out[1]), O._p(out[2]), ctypes.c_int(symmetry))
    return out


# the shift's parities for mass^i; the state's for chi .. A~zz (bssn_class.C:209-232)
MASS_SOA = [(-1.0, 1.0, 1.0), (1.0, -1.0, 1.0), (1.0, 1.0, -1.0)]
STATE_SOA = {0: (1, 1, 1), 1: (1, 1, 1), 2: (1, 1, 1), 3: (-1, -1, 1), 4: (-1, 1, -1), 5: (1, 1, 1), 6: (1, -1, -1),
             7: (1, 1, 1), 8: (1, 1, 1), 9: (-1, -1, 1), 10: (-1, 1, -1), 11: (1, 1, 1), 12: (1, -1, -1),
             13: (1, 1, 1)}


def surf_masspang(rex, values, nquarter, symmetry):
    """surface_integral.C:2247-2512 (GaussInt) given the 17 interpolated values
    per sphere point (mass^x, mass^y, mass^z, chi, trK, gxx .. gzz, Axx .. Azz):
    [mass, Px, Py, Pz, Sx, Sy, Sz]."""
    ct, wt, n_theta, n_phi, dphi, pts = sphere(nquarter, symmetry)
    factor = {0: 1, 1: 2, 2: 8}[symmetry]
    f1o8 = 0.125
    mass = ax = ay = az = px = py = pz = 0.0
    for n in range(n_theta * n_phi):
        i = n // n_phi
        nx, ny, nz = pts[n]
        X, Y, Z = rex * nx, rex * ny, rex * nz
        s = values[n]
        Chi, TRK = s[3], s[4]
        Gxx, Gxy, Gxz, Gyy, Gyz, Gzz = s[5] + 1.0, s[6], s[7], s[8] + 1.0, s[9], s[10] + 1.0
        axx, axy, axz, ayy, ayz, azz = s[11], s[12], s[13], s[14], s[15], s[16]
        Chi = 1.0 / (1.0 + Chi)
        Psi = Chi * math.sqrt(Chi)
        mass = mass + (s[0] * nx + s[1] * ny + s[2] * nz) * wt[i]
        gupzz = Gxx * Gyy * Gzz + Gxy * Gyz * Gxz + Gxz * Gxy * Gyz - Gxz * Gyy * Gxz - Gxy * Gxy * Gzz - Gxx * Gyz * Gyz
        gupxx = (Gyy * Gzz - Gyz * Gyz) / gupzz
        gupxy = -(Gxy * Gzz - Gyz * Gxz) / gupzz
        gupxz = (Gxy * Gyz - Gyy * Gxz) / gupzz
        gupyy = (Gxx * Gzz - Gxz * Gxz) / gupzz
        gupyz = -(Gxx * Gyz - Gxy * Gxz) / gupzz
        gupzz = (Gxx * Gyy - Gxy * Gxy) / gupzz
        aupxx = gupxx * axx + gupxy * axy + gupxz * axz
        aupxy = gupxx * axy + gupxy * ayy + gupxz * ayz
        aupxz = gupxx * axz + gupxy * ayz + gupxz * azz
        aupyx = gupxy * axx + gupyy * axy + gupyz * axz
        aupyy = gupxy * axy + gupyy * ayy + gupyz * ayz
        aupyz = gupxy * axz + gupyy * ayz + gupyz * azz
        aupzx = gupxz * axx + gupyz * axy + gupzz * axz
        aupzy = gupxz * axy + gupyz * ayy + gupzz * ayz
        aupzz = gupxz * axz + gupyz * ayz + gupzz * azz
        if symmetry == 0:
            ax = ax + f1o8 * Psi * (nx * (Y * aupxz - Z * aupxy) + ny * (Y * aupyz - Z * aupyy) +
                                    nz * (Y * aupzz - Z * aupzy)) * wt[i]
            ay = ay + f1o8 * Psi * (nx * (Z * aupxx - X * aupxz) + ny * (Z * aupyx - X * aupyz) +
                                    nz * (Z * aupzx - X * aupzz)) * wt[i]
        if symmetry in (0, 1):
            az = az + f1o8 * Psi * (nx * (X * aupxy - Y * aupxx) + ny * (X * aupyy - Y * aupyx) +
                                    nz * (X * aupzy - Y * aupzx)) * wt[i]
        axx = Chi * (axx + Gxx * TRK / 3.0)
        axy = Chi * (axy + Gxy * TRK / 3.0)
        axz = Chi * (axz + Gxz * TRK / 3.0)
        ayy = Chi * (ayy + Gyy * TRK / 3.0)
        ayz = Chi * (ayz + Gyz * TRK / 3.0)
        azz = Chi * (azz + Gzz * TRK / 3.0)
        axx = axx - TRK
        ayy = ayy - TRK
        azz = azz - TRK
        if symmetry in (0, 1):
            px = px + f1o8 * Psi * (nx * axx + ny * axy + nz * axz) * wt[i]
            py = py + f1o8 * Psi * (nx * axy + ny * ayy + nz * ayz) * wt[i]
        if symmetry == 0:
            pz = pz + f1o8 * Psi * (nx * axz + ny * ayz + nz * azz) * wt[i]
    sc = lambda v: v * rex * rex * dphi * (1.0 / PI) * factor   # noqa: E731
    return [mass * rex * rex * dphi * factor, sc(px), sc(py), sc(pz), sc(ax), sc(ay), sc(az)]


def adm_extract(H, level, states, rex, nquarter, symmetry=0):
    """surf_MassPAng on a level: admmass_bssn per block (not synchronised),
    the 17 values interpolated on the sphere, the sums."""
    ids = [bi for p in H.levels[level] for bi in p.blocks]
    comb = {}
    for bi in ids:
        b = H.blocks[bi]
        X, Y, Z = H.coords(b)
        comb[bi] = np.concatenate([admmass(X, Y, Z, states[bi], symmetry), states[bi][:14]])
    _, _, _, _, _, pts = sphere(nquarter, symmetry)
    P = OI.hierarchy_patches(H, level, comb)
    soas = MASS_SOA + [STATE_SOA[k] for k in range(14)]
    vals, found = OI.interp_points(P, [(rex * a, rex * b, rex * c) for a, b, c in pts], list(range(17)), soas,
                                   symmetry)
    if not all(found):
        raise ValueError("a sphere point lies outside the level")
    return surf_masspang(rex, vals, nquarter, symmetry)
