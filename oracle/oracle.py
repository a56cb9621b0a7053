"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a plain-C restatement of the AMSS-NCKU Fortran kernels on the
BSSN evolution path (see oracle_common.h for the parity status: unpinned).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.

Block fields are numpy float64 arrays of shape (ex[2], ex[1], ex[0]) in C order,
which is the reference's Fortran order (i fastest).  A block state is an array
of shape (24, ex[2], ex[1], ex[0]) in the state order of bssn_rhs.f90:6-11.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_amss.so")

STATE_NAMES = ["chi", "trK", "gxx", "gxy", "gxz", "gyy", "gyz", "gzz",
               "Axx", "Axy", "Axz", "Ayy", "Ayz", "Azz", "Gamx", "Gamy", "Gamz",
               "Lap", "betax", "betay", "betaz", "dtSfx", "dtSfy", "dtSfz"]
GAMMA_NAMES = ["Gamxxx", "Gamxxy", "Gamxxz", "Gamxyy", "Gamxyz", "Gamxzz",
               "Gamyxx", "Gamyxy", "Gamyxz", "Gamyyy", "Gamyyz", "Gamyzz",
               "Gamzxx", "Gamzxy", "Gamzxz", "Gamzyy", "Gamzyz", "Gamzzz"]
RICCI_NAMES = ["Rxx", "Rxy", "Rxz", "Ryy", "Ryz", "Rzz"]
CONSTRAINT_NAMES = ["ham", "movx", "movy", "movz", "Gmx", "Gmy", "Gmz"]

_lib = None
_DP = ctypes.POINTER(ctypes.c_double)


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_compute_rhs_bssn.restype = ctypes.c_int
        _lib.oracle_bssn_step_single.restype = ctypes.c_int
        _lib.oracle_l2normhelper.restype = ctypes.c_double
        _lib.oracle_rungekutta4_rout.restype = ctypes.c_int
        _lib.oracle_sommerfeld_rout.restype = ctypes.c_int
        _lib.oracle_bssn_propspeed.restype = ctypes.c_double
    return _lib


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def _ex(shape):
    return (ctypes.c_int * 3)(shape[-1], shape[-2], shape[-3])


def cell_coords(lo, hi, n):
    """Block.C:48-52 (Cell): X[j] = bbox_lo + (j + 0.5) * h, h = (hi - lo) / n."""
    h = (hi - lo) / n
    return np.array([lo + (j + 0.5) * h for j in range(n)], dtype=np.float64)


def compute_rhs_bssn(X, Y, Z, state, matter=None, symmetry=0, lev=0, eps=0.1, co=1, T=0.0):
    """bssn_rhs.f90:5-1184.  Returns (gont, rhs[24], gamma[18], ricci[6], cons[7]).

    `state` is modified in place only where the Fortran's intent(inout) allows
    (it is not, in fact, written)."""
    state = np.ascontiguousarray(state, dtype=np.float64)
    shp = state.shape[1:]
    ex = _ex(shp)
    rhs = np.zeros((24,) + shp)
    gam = np.zeros((18,) + shp)
    ric = np.zeros((6,) + shp)
    cons = np.zeros((7,) + shp)
    if matter is None:
        matter = np.zeros((10,) + shp)
    matter = np.ascontiguousarray(matter, dtype=np.float64)
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    args = [ex, ctypes.c_double(T), _p(X), _p(Y), _p(Z)]
    args += [_p(state[f]) for f in range(24)]
    args += [_p(rhs[f]) for f in range(24)]
    args += [_p(matter[f]) for f in range(10)]
    args += [_p(gam[f]) for f in range(18)]
    args += [_p(ric[f]) for f in range(6)]
    args += [_p(cons[f]) for f in range(7)]
    args += [ctypes.c_int(symmetry), ctypes.c_int(lev), ctypes.c_double(eps), ctypes.c_int(co)]
    gont = lib().oracle_compute_rhs_bssn(*args)
    return gont, rhs, gam, ric, cons


def compute_rhs_z4c(X, Y, Z, state, matter=None, symmetry=0, lev=0, eps=0.1, T=0.0):
    """Z4c_rhs.f90:126-1295 (state of 25 fields, Theta last).  Returns
    (gont, rhs[25], gamma[18], ricci[6], cons[7]); the constraints are always
    computed (the Fortran ignores co)."""
    state = np.ascontiguousarray(state, dtype=np.float64)
    shp = state.shape[1:]
    ex = _ex(shp)
    rhs = np.zeros((25,) + shp)
    gam = np.zeros((18,) + shp)
    ric = np.zeros((6,) + shp)
    cons = np.zeros((7,) + shp)
    if matter is None:
        matter = np.zeros((10,) + shp)
    matter = np.ascontiguousarray(matter, dtype=np.float64)
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    args = [ex, ctypes.c_double(T), _p(X), _p(Y), _p(Z)]
    args += [_p(state[f]) for f in range(25)]
    args += [_p(rhs[f]) for f in range(25)]
    args += [_p(matter[f]) for f in range(10)]
    args += [_p(gam[f]) for f in range(18)]
    args += [_p(ric[f]) for f in range(6)]
    args += [_p(cons[f]) for f in range(7)]
    args += [ctypes.c_int(symmetry), ctypes.c_int(lev), ctypes.c_double(eps), ctypes.c_int(0)]
    gont = lib().oracle_compute_rhs_z4c(*args)
    return gont, rhs, gam, ric, cons


def fderivs(X, Y, Z, f, soa=(1.0, 1.0, 1.0), symmetry=0):
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = [np.zeros_like(f) for _ in range(3)]
    lib().oracle_fderivs(_ex(f.shape), _p(f), *[_p(o) for o in out], _p(X), _p(Y), _p(Z),
                         *[ctypes.c_double(s) for s in soa], ctypes.c_int(symmetry))
    return out


def fdderivs(X, Y, Z, f, soa=(1.0, 1.0, 1.0), symmetry=0):
    """Returns fxx, fxy, fxz, fyy, fyz, fzz."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = [np.zeros_like(f) for _ in range(6)]
    lib().oracle_fdderivs(_ex(f.shape), _p(f), *[_p(o) for o in out], _p(X), _p(Y), _p(Z),
                          *[ctypes.c_double(s) for s in soa], ctypes.c_int(symmetry))
    return out


def lopsided(X, Y, Z, f, beta, soa=(1.0, 1.0, 1.0), symmetry=0):
    """lopsidediff.f90:186-488 added to a zero right-hand side: the upwinded
    advection beta^i d_i f."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    r = np.zeros_like(f)
    b = [np.ascontiguousarray(x, dtype=np.float64) for x in beta]
    s = np.ascontiguousarray(soa, dtype=np.float64)
    lib().oracle_lopsided(_ex(f.shape), _p(X), _p(Y), _p(Z), _p(f), _p(r), _p(b[0]), _p(b[1]), _p(b[2]),
                          ctypes.c_int(symmetry), _p(s))
    return r


def kodis(X, Y, Z, f, soa=(1.0, 1.0, 1.0), symmetry=0, eps=0.1):
    """kodiss.f90:120-216 added to a zero right-hand side."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    r = np.zeros_like(f)
    s = np.ascontiguousarray(soa, dtype=np.float64)
    lib().oracle_kodis(_ex(f.shape), _p(X), _p(Y), _p(Z), _p(f), _p(r), _p(s), ctypes.c_int(symmetry),
                       ctypes.c_double(eps))
    return r


def enforce_ga(state):
    """In place on state[2:14] (enforce_algebra.f90:72-133)."""
    ex = _ex(state.shape[1:])
    lib().oracle_enforce_ga(ex, *[_p(state[f]) for f in range(2, 14)])


def rungekutta4_rout(dT, f0, f1, f_rhs, rk4):
    return lib().oracle_rungekutta4_rout(_ex(f0.shape), ctypes.c_double(dT), _p(f0), _p(f1), _p(f_rhs),
                                         ctypes.c_int(rk4))


def lowerboundset(chi, tiny):
    lib().oracle_lowerboundset(_ex(chi.shape), _p(chi), ctypes.c_double(tiny))


def sommerfeld_routbam(X, Y, Z, bbox, f_rhs, f0, velocity, soa, symmetry=0):
    lib().oracle_sommerfeld_routbam(_ex(f0.shape), _p(X), _p(Y), _p(Z), *[ctypes.c_double(b) for b in bbox],
                                    _p(f_rhs), _p(f0), ctypes.c_double(velocity),
                                    _p(np.asarray(soa, dtype=np.float64)), ctypes.c_int(symmetry))


def sommerfeld_rout_freeze(X, Y, Z, bbox, f0, f, symmetry=0):
    return lib().oracle_sommerfeld_rout(_ex(f0.shape), _p(X), _p(Y), _p(Z), *[ctypes.c_double(b) for b in bbox],
                                        _p(f0), _p(f), ctypes.c_int(symmetry), ctypes.c_int(1))


def get_lousto_nbhs(X, Y, Z, masses, positions, momenta=None, spins=None):
    """initial_puncture.f90:1970-2202: the 24-field state of N punctures."""
    ex = (len(X), len(Y), len(Z))
    st = np.zeros((24, ex[2], ex[1], ex[0]))
    m = np.ascontiguousarray(masses, dtype=np.float64).reshape(-1)
    porg = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
    zeros = np.zeros(3 * len(m))
    pmom = zeros if momenta is None else np.ascontiguousarray(momenta, dtype=np.float64).reshape(-1)
    spin = zeros if spins is None else np.ascontiguousarray(spins, dtype=np.float64).reshape(-1)
    ptrs = (_DP * 24)(*[_p(st[f]) for f in range(24)])
    lib().oracle_get_lousto_nbhs((ctypes.c_int * 3)(*ex), _p(np.ascontiguousarray(X)), _p(np.ascontiguousarray(Y)),
                                 _p(np.ascontiguousarray(Z)), ptrs, _p(m), _p(porg), _p(pmom), _p(spin),
                                 ctypes.c_int(len(m)))
    return st


def brill_lindquist(X, Y, Z, masses, positions):
    """get_lousto_nbhs with zero momenta and spins: the Brill-Lindquist data."""
    return get_lousto_nbhs(X, Y, Z, masses, positions)


def l2normhelper(X, Y, Z, bbox, f, gw):
    return lib().oracle_l2normhelper(_ex(f.shape), _p(X), _p(Y), _p(Z), *[ctypes.c_double(b) for b in bbox],
                                     _p(np.ascontiguousarray(f)), ctypes.c_int(gw))


def propspeed(field):
    return lib().oracle_bssn_propspeed(ctypes.c_int(field))


BSSN_SOA = np.array([
    [1, 1, 1], [1, 1, 1], [1, 1, 1], [-1, -1, 1], [-1, 1, -1], [1, 1, 1], [1, -1, -1], [1, 1, 1],
    [1, 1, 1], [-1, -1, 1], [-1, 1, -1], [1, 1, 1], [1, -1, -1], [1, 1, 1],
    [-1, 1, 1], [1, -1, 1], [1, 1, -1], [1, 1, 1], [-1, 1, 1], [1, -1, 1], [1, 1, -1],
    [-1, 1, 1], [1, -1, 1], [1, 1, -1]], dtype=np.float64)


def bssn_step_single(X, Y, Z, bbox, state, dT, eps=0.1, chitiny=1e-5 - 1.0, symmetry=0, T=0.0):
    """One RK4 step of one block that is the whole level-0 patch, in place."""
    ptrs = (_DP * 24)(*[_p(state[f]) for f in range(24)])
    return lib().oracle_bssn_step_single(_ex(state.shape[1:]), _p(X), _p(Y), _p(Z),
                                         _p(np.asarray(bbox, dtype=np.float64)), ptrs, ctypes.c_double(dT),
                                         ctypes.c_double(eps), ctypes.c_double(chitiny), ctypes.c_int(symmetry),
                                         ctypes.c_double(T))


def single_block_setup(n_interior, lo, hi, ghosts, masses, positions, noise=0.0, seed=1):
    """A uniform cell-centred block of n_interior^3 cells on [lo, hi]^3 plus
    `ghosts` cells each side, treated as one level-0 patch (its outer cells are
    ordinary evolved cells with reduced stencils).  Brill-Lindquist data plus
    seeded uniform noise U(-noise, noise) on every field, drawn with
    numpy.random.default_rng(seed) field by field in state order."""
    h = (hi - lo) / n_interior
    n = n_interior + 2 * ghosts
    a_lo, a_hi = lo - ghosts * h, hi + ghosts * h
    X = cell_coords(a_lo, a_hi, n)
    st = brill_lindquist(X, X, X, masses, positions)
    if noise > 0:
        rng = np.random.default_rng(seed)
        for f in range(24):
            st[f] += rng.uniform(-noise, noise, size=st[f].shape)
    bbox = (a_lo, a_lo, a_lo, a_hi, a_hi, a_hi)
    return X, st, bbox, h
