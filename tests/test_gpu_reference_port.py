"""Pins the oracle to code built from the reference itself.

oracle/build_ref.py compiles the reference's 2015 CUDA port of
compute_rhs_bssn (AMSS_NCKU_source/bssn_gpu.cu, gpu_rhs) with the header its
own generator writes for the evolution path (GAUGE 0, Cell, ghost_width 3),
into oracle/_ref/libref_bssn_gpu.so.  Here that library, the oracle (the C
restatement of bssn_rhs.f90) and the product's drop-in compute_rhs_bssn_ run on
the same vacuum blocks; every output -- the 24 right-hand sides, the 18
Christoffel symbols, the 6 Ricci components and, with co = 0, the 7
constraint residuals -- must agree to <= 1e-12 of the field's max-norm over
the points at least 3 cells from every face.

Nearer the faces the port is not a restatement of the Fortran, so it is not
compared there: its second derivatives gate the 4th/2nd-order fallback per
direction pair instead of jointly over all three directions
(bssn_gpu.cu:286-370 against diff_new.f90:1486-1520), and the derivative
arrays it reuses are cleared with a byte count that host code reads from a
__constant__ symbol (bssn_gpu.cu:375-380, :444-446; nvcc warns that the host
sees a shadow holding 0), i.e. not at all, so its outermost planes keep earlier
values where the Fortran writes 0.  The port also zeroes
the matter sources itself (bssn_gpu.cu:2421-2430), so the blocks are vacuum.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from amss_b200 import dropin as D

from helpers import generic_state

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libref_bssn_gpu.so")
TOL = 1e-12


def _port(X, Y, Z, st, eps, co, symmetry=0):
    """gpu_rhs twice: called as the step (the right-hand sides come back)
    and as the constraint output (the Christoffels, Ricci and residuals)."""
    rhs = _port_call(0, X, Y, Z, st, eps, co, symmetry)[0]
    aux = _port_call(1, X, Y, Z, st, eps, co, symmetry)[1:]
    return [rhs] + aux


def _port_call(calledby, X, Y, Z, st, eps, co, symmetry=0):
    lib = ctypes.CDLL(LIB)
    P = ctypes.POINTER(ctypes.c_double)
    st = np.ascontiguousarray(st)
    shp = st.shape[1:]
    out = [np.zeros((k,) + shp) for k in (24, 18, 6, 7)]
    matter = np.zeros((10,) + shp)
    p = lambda a: a.ctypes.data_as(P)   # noqa: E731
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    args = [ctypes.c_int(calledby), (ctypes.c_int * 3)(shp[2], shp[1], shp[0]), ctypes.byref(ctypes.c_double(0.0)),
            p(X), p(Y), p(Z)]
    args += [p(st[f]) for f in range(24)] + [p(out[0][f]) for f in range(24)]
    args += [p(matter[f]) for f in range(10)]
    args += [p(a[f]) for a in out[1:] for f in range(a.shape[0])]
    args += [ctypes.byref(ctypes.c_int(symmetry)), ctypes.byref(ctypes.c_int(0)),
             ctypes.byref(ctypes.c_double(eps)), ctypes.byref(ctypes.c_int(co))]
    rc = lib.ref_gpu_rhs(*args)
    assert rc == 0
    return out


def _interior_errs(a, b, co):
    """Per output group and field: max |a - b| over points >= 3 cells from every
    face, over max |b| there."""
    errs = {}
    groups = ("rhs", "gamma", "ricci", "cons") if co == 0 else ("rhs", "gamma", "ricci")
    for g, name in enumerate(groups):
        for f in range(a[g].shape[0]):
            x = a[g][f][3:-3, 3:-3, 3:-3]
            y = b[g][f][3:-3, 3:-3, 3:-3]
            den = np.abs(y).max()
            errs[(name, f)] = np.abs(x - y).max() / den if den > 0 else np.abs(x - y).max()
    return errs


@pytest.mark.skipif(not os.path.exists(LIB), reason="reference port not built (python oracle/build_ref.py)")
@pytest.mark.parametrize("case", ["bl", "generic"])
def test_oracle_and_product_match_the_reference_port(case):
    if case == "bl":
        X, st, bbox, h = O.single_block_setup(18, -4.5, 4.5, 3, [1.0], [[0.1, 0.05, 0.02]], noise=1e-8, seed=3)
        Y = Z = X
        eps = 0.1
    else:
        X = O.cell_coords(-2.0, 2.5, 22)
        Y = O.cell_coords(-1.5, 2.0, 20)
        Z = O.cell_coords(-3.0, 1.0, 24)
        st = generic_state(X, Y, Z, seed=4)
        eps = 0.2
    ref = _port(X, Y, Z, st, eps, co=0)
    orc = O.compute_rhs_bssn(X, Y, Z, st, eps=eps, co=0)
    got = D.compute_rhs_bssn(X, Y, Z, st, eps=eps, co=0)
    assert orc[0] == got[0] == 0
    e_orc = _interior_errs(list(orc[1:]), ref, 0)
    e_got = _interior_errs(list(got[1:]), ref, 0)
    bad = {k: (e_orc[k], e_got[k]) for k in e_orc if e_orc[k] > TOL or e_got[k] > TOL}
    assert not bad, sorted(bad.items(), key=lambda kv: -max(kv[1]))[:10]
