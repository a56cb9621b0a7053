"""Host-side mirror of the reference's per-block kernel calls.

Each function takes the arguments the reference's C++ driver passes to the
Fortran kernel of the same name (bssn_class.C:3052-3156) -- coordinate arrays,
Fortran-order field arrays, symmetry flag, dissipation, RK4 counter -- and runs
it through the drop-in C ABI of libamss_b200.so on the GPU.

Block fields are numpy float64 arrays of shape (ex[2], ex[1], ex[0]) in C
order, which is the reference's Fortran order (i fastest); a block state is
(24, ex[2], ex[1], ex[0]) in the state order of bssn_rhs.f90:6-11.
"""
import ctypes

import numpy as np

from ._lib import _DP, AmssError, check, lib

STATE_NAMES = ["chi", "trK", "gxx", "gxy", "gxz", "gyy", "gyz", "gzz",
               "Axx", "Axy", "Axz", "Ayy", "Ayz", "Azz", "Gamx", "Gamy", "Gamz",
               "Lap", "betax", "betay", "betaz", "dtSfx", "dtSfy", "dtSfz"]


def _p(a):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise AmssError("arrays must be C-contiguous float64")
    return a.ctypes.data_as(_DP)


def _ex(shape):
    return (ctypes.c_int * 3)(shape[-1], shape[-2], shape[-3])


def compute_rhs_bssn(X, Y, Z, state, matter=None, symmetry=0, lev=0, eps=0.1, co=1, T=0.0):
    """compute_rhs_bssn (bssn_rhs.f90:5-1184) on the GPU.

    Returns (gont, rhs[24], gamma[18], ricci[6], cons[7]); gont == 1 means the
    input held a NaN and, as in the reference, no output was written."""
    state = np.ascontiguousarray(state, dtype=np.float64)
    shp = state.shape[1:]
    rhs = np.zeros((24,) + shp)
    gam = np.zeros((18,) + shp)
    ric = np.zeros((6,) + shp)
    cons = np.zeros((7,) + shp)
    if matter is None:
        matter = np.zeros((10,) + shp)
    matter = np.ascontiguousarray(matter, dtype=np.float64)
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    args = [_ex(shp), ctypes.byref(ctypes.c_double(T)), _p(X), _p(Y), _p(Z)]
    args += [_p(state[f]) for f in range(24)]
    args += [_p(rhs[f]) for f in range(24)]
    args += [_p(matter[f]) for f in range(10)]
    args += [_p(gam[f]) for f in range(18)]
    args += [_p(ric[f]) for f in range(6)]
    args += [_p(cons[f]) for f in range(7)]
    args += [ctypes.byref(ctypes.c_int(symmetry)), ctypes.byref(ctypes.c_int(lev)),
             ctypes.byref(ctypes.c_double(eps)), ctypes.byref(ctypes.c_int(co))]
    gont = check(lib().compute_rhs_bssn_(*args), "compute_rhs_bssn_")
    return gont, rhs, gam, ric, cons


def compute_rhs_z4c(X, Y, Z, state, matter=None, symmetry=0, lev=0, eps=0.1, T=0.0):
    """compute_rhs_Z4c (Z4c_rhs.f90:126-1295) on the GPU; state of 25 fields
    (Theta last).  Returns (gont, rhs[25], gamma[18], ricci[6], cons[7]); the
    constraints are always computed."""
    state = np.ascontiguousarray(state, dtype=np.float64)
    shp = state.shape[1:]
    out = [np.zeros((k,) + shp) for k in (25, 18, 6, 7)]
    matter = np.zeros((10,) + shp) if matter is None else np.ascontiguousarray(matter, dtype=np.float64)
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    args = [_ex(shp), ctypes.byref(ctypes.c_double(T)), _p(X), _p(Y), _p(Z)]
    args += [_p(state[f]) for f in range(25)] + [_p(out[0][f]) for f in range(25)]
    args += [_p(matter[f]) for f in range(10)]
    args += [_p(a[f]) for a in out[1:] for f in range(a.shape[0])]
    args += [ctypes.byref(ctypes.c_int(symmetry)), ctypes.byref(ctypes.c_int(lev)),
             ctypes.byref(ctypes.c_double(eps)), ctypes.byref(ctypes.c_int(0))]
    gont = check(lib().compute_rhs_z4c_(*args), "compute_rhs_z4c_")
    return (gont,) + tuple(out)


def compute_rhs_bssn_noalloc(X, Y, Z, state, matter=None, symmetry=0, lev=0, eps=0.1, co=1, T=0.0):
    """compute_rhs_bssn through amss_compute_rhs_bssn_noalloc: the same
    kernel with no device allocation; blocks of at most
    AMSS_NOALLOC_MAX_POINTS (32768) points; calls must not overlap.  Same
    return value as compute_rhs_bssn."""
    state = np.ascontiguousarray(state, dtype=np.float64)
    shp = state.shape[1:]
    out = [np.zeros((k,) + shp) for k in (24, 18, 6, 7)]
    matter = np.zeros((10,) + shp) if matter is None else np.ascontiguousarray(matter, dtype=np.float64)
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    args = [_ex(shp), ctypes.byref(ctypes.c_double(T)), _p(X), _p(Y), _p(Z)]
    args += [_p(state[f]) for f in range(24)] + [_p(out[0][f]) for f in range(24)]
    args += [_p(matter[f]) for f in range(10)]
    args += [_p(a[f]) for a in out[1:] for f in range(a.shape[0])]
    args += [ctypes.byref(ctypes.c_int(symmetry)), ctypes.byref(ctypes.c_int(lev)),
             ctypes.byref(ctypes.c_double(eps)), ctypes.byref(ctypes.c_int(co))]
    gont = check(lib().amss_compute_rhs_bssn_noalloc(*args), "amss_compute_rhs_bssn_noalloc")
    return (gont,) + tuple(out)


def rungekutta4_rout(dT, f0, f1, f_rhs, rk4):
    """rungekutta4_rout (rungekutta4_rout.f90:94-139), f1 and f_rhs in place."""
    return check(lib().rungekutta4_rout_(_ex(f0.shape), ctypes.byref(ctypes.c_double(dT)), _p(f0), _p(f1),
                                         _p(f_rhs), ctypes.byref(ctypes.c_int(rk4))), "rungekutta4_rout_")


def _scalars(*vals):
    return [ctypes.byref(ctypes.c_double(v)) for v in vals]


def sommerfeld_routbam(X, Y, Z, bbox, f_rhs, f0, velocity, soa, symmetry=0):
    """sommerfeld_routbam (sommerfeld_rout.f90:223-449), f_rhs in place."""
    soa = np.ascontiguousarray(soa, dtype=np.float64)
    lib().sommerfeld_routbam_(_ex(f0.shape), _p(X), _p(Y), _p(Z), *_scalars(*bbox), _p(f_rhs), _p(f0),
                              ctypes.byref(ctypes.c_double(velocity)), _p(soa),
                              ctypes.byref(ctypes.c_int(symmetry)))


def sommerfeld_rout_freeze(X, Y, Z, bbox, f0, f, symmetry=0, dT=0.0):
    """sommerfeld_rout with precor == 1 (sommerfeld_rout.f90:122-139), f in place."""
    dummy = np.zeros(1)
    soa = np.ones(3)
    lib().sommerfeld_rout_(_ex(f0.shape), _p(X), _p(Y), _p(Z), *_scalars(*bbox), ctypes.byref(ctypes.c_double(dT)),
                           _p(dummy), _p(dummy), _p(f0), _p(f), _p(soa), ctypes.byref(ctypes.c_int(symmetry)),
                           ctypes.byref(ctypes.c_int(1)))


def enforce_ga(state):
    """enforce_ga (enforce_algebra.f90:72-133) in place on state[2:14]."""
    lib().enforce_ga_(_ex(state.shape[1:]), *[_p(state[f]) for f in range(2, 14)])


def lowerboundset(chi, tiny):
    """lowerboundset (fmisc.f90:1644-1657) in place."""
    lib().lowerboundset_(_ex(chi.shape), _p(chi), ctypes.byref(ctypes.c_double(tiny)))


def get_lousto_nbhs(X, Y, Z, masses, positions, momenta=None, spins=None):
    """get_lousto_nbhs (initial_puncture.f90:1970-2202) on the GPU: the 24-field
    state (offsets) of N punctures; zero momenta and spins give Brill-Lindquist."""
    X, Y, Z = (np.ascontiguousarray(a, dtype=np.float64) for a in (X, Y, Z))
    m = np.ascontiguousarray(masses, dtype=np.float64).reshape(-1)
    n = len(m)
    porg = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
    pmom = np.zeros(3 * n) if momenta is None else np.ascontiguousarray(momenta, dtype=np.float64).reshape(-1)
    spin = np.zeros(3 * n) if spins is None else np.ascontiguousarray(spins, dtype=np.float64).reshape(-1)
    if porg.size != 3 * n or pmom.size != 3 * n or spin.size != 3 * n:
        raise AmssError("positions, momenta and spins need 3 values per puncture")
    st = np.empty((24, len(Z), len(Y), len(X)))
    check(lib().get_lousto_nbhs_((ctypes.c_int * 3)(len(X), len(Y), len(Z)), _p(X), _p(Y), _p(Z),
                                 *[_p(st[f]) for f in range(24)], _p(m), _p(porg), _p(pmom), _p(spin),
                                 ctypes.byref(ctypes.c_int(n))), "get_lousto_nbhs_")
    return st


def lousto_vjp(X, Y, Z, masses, positions, state_b):
    """Adjoints of the Brill-Lindquist masses and positions for the state
    adjoint state_b (24, ex[2], ex[1], ex[0]): (dmass[N], dpos[N, 3])."""
    X, Y, Z = (np.ascontiguousarray(a, dtype=np.float64) for a in (X, Y, Z))
    m = np.ascontiguousarray(masses, dtype=np.float64).reshape(-1)
    porg = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
    chi_b = np.ascontiguousarray(state_b[0], dtype=np.float64)
    lap_b = np.ascontiguousarray(state_b[17], dtype=np.float64)
    dm = np.zeros(len(m))
    dp = np.zeros(3 * len(m))
    check(lib().amss_lousto_vjp((ctypes.c_int * 3)(len(X), len(Y), len(Z)), _p(X), _p(Y), _p(Z), len(m), _p(m),
                                _p(porg), _p(chi_b), _p(lap_b), _p(dm), _p(dp)), "amss_lousto_vjp")
    return dm, dp.reshape(-1, 3)
