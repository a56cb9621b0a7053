"""The straight-line programs the adjoint is generated from (no GPU).

gen/tape_*.txt are recordings of the kernels' own point functions by
gen/trace_rhs.cpp: the split-form right-hand side (bssn_rhs_point, BSSN and
Z4c), the Hamiltonian constraint and enforce_ga_point.  Fed with the stencil
terms the oracle's fderivs / fdderivs / lopsided / kodis produce, a tape must
give the oracle's values; its reverse sweep must agree with central finite
differences of the tape.
"""
import os
import sys

import numpy as np
import pytest

import oracle as O

from helpers import generic_state

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "nr-amssncku_b200", "gen"))
import tape as TP  # noqa: E402

SOA = [(1, 1, 1), (1, 1, 1), (1, 1, 1), (-1, -1, 1), (-1, 1, -1), (1, 1, 1), (1, -1, -1), (1, 1, 1),
       (1, 1, 1), (-1, -1, 1), (-1, 1, -1), (1, 1, 1), (1, -1, -1), (1, 1, 1),
       (-1, 1, 1), (1, -1, 1), (1, 1, -1), (1, 1, 1), (-1, 1, 1), (1, -1, 1), (1, 1, -1),
       (-1, 1, 1), (1, -1, 1), (1, 1, -1), (1, 1, 1)]
KIND0 = [0, 17, 18, 19, 20, 2, 3, 4, 5, 6, 7]   # gradient + Hessian + adv
KIND1 = [1, 14, 15, 16, 24]                     # gradient + adv


def nslots(f):
    return 10 if f in KIND0 else (4 if f in KIND1 else 1)


def doff(f):
    return sum(nslots(g) for g in range(f))


def stencil_terms(X, Y, Z, st, eps, z4c):
    """D slots as the stencil pass stores them, from the oracle's stencils."""
    nf = st.shape[0]
    beta = st[18:21]
    d = {}
    for f in range(nf):
        o = doff(f)
        if f in KIND0 or f in KIND1:
            g = O.fderivs(X, Y, Z, st[f], SOA[f])
            for m in range(3):
                d[o + m] = g[m]
        if f in KIND0:
            h = O.fdderivs(X, Y, Z, st[f], SOA[f])
            for m in range(6):
                d[o + 3 + m] = h[m]
        diag = f in (2, 5, 7)
        adv = O.lopsided(X, Y, Z, st[f] + (1.0 if diag else 0.0), beta, SOA[f])
        adv = adv + O.kodis(X, Y, Z, st[f] + (1.0 if (diag and z4c) else 0.0), SOA[f], eps=eps)
        d[o + nslots(f) - 1] = adv
    return d


@pytest.mark.parametrize("z4c", [False, True])
def test_tape_forward_matches_oracle_rhs(z4c):
    X = O.cell_coords(-2.0, 2.5, 18)
    Y = O.cell_coords(-1.5, 2.0, 16)
    Z = O.cell_coords(-3.0, 1.0, 14)
    st = generic_state(X, Y, Z, seed=7)
    if z4c:
        z, y, x = np.meshgrid(Z, Y, X, indexing="ij")
        st = np.concatenate([st, (2e-3 * np.sin(0.7 * x) * np.cos(0.5 * y + z))[None]])
        ref = O.compute_rhs_z4c(X, Y, Z, st, eps=0.1)[1]
    else:
        ref = O.compute_rhs_bssn(X, Y, Z, st, eps=0.1, co=1)[1]
    tp = TP.Tape(os.path.join(HERE, "..", "nr-amssncku_b200", "gen", "tape_z4c.txt" if z4c else "tape_bssn.txt"))
    out = tp.evaluate({f: st[f] for f in range(st.shape[0])}, stencil_terms(X, Y, Z, st, 0.1, z4c))
    assert sorted(out) == list(range(st.shape[0]))
    # stencils are gated identically in the tape's inputs, so compare every point
    for f in range(st.shape[0]):
        den = np.abs(ref[f]).max()
        err = np.abs(out[f] - ref[f]).max() / den
        assert err <= 1e-12, (f, err)


def _tape(name):
    return TP.Tape(os.path.join(HERE, "..", "nr-amssncku_b200", "gen", f"tape_{name}.txt"))


def test_ham_tape_matches_oracle_constraint():
    X = O.cell_coords(-2.0, 2.5, 18)
    Y = O.cell_coords(-1.5, 2.0, 16)
    Z = O.cell_coords(-3.0, 1.0, 14)
    st = generic_state(X, Y, Z, seed=9)
    ref = O.compute_rhs_bssn(X, Y, Z, st, eps=0.1, co=0)[4][0]
    out = _tape("ham").evaluate({f: st[f] for f in range(24)}, stencil_terms(X, Y, Z, st, 0.1, False))
    assert np.abs(out[99] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_enforce_tape_matches_oracle():
    rng = np.random.default_rng(5)
    st = np.zeros((24, 4, 5, 6))
    for f in range(2, 14):
        st[f] = rng.uniform(-0.1, 0.1, st.shape[1:])
    ref = st.copy()
    O.enforce_ga(ref)
    out = _tape("enforce").evaluate({m: st[2 + m] for m in range(12)}, {})
    for m in range(12):
        assert np.abs(out[m] - ref[2 + m]).max() <= 1e-14, m


@pytest.mark.parametrize("name", ["bssn", "z4c", "ham", "enforce"])
def test_tape_reverse_sweep_matches_finite_differences(name):
    """<rb, J dx> from central differences of the tape equals <J^T rb, dx>."""
    tp = _tape(name)
    rng = np.random.default_rng(3)
    npt = 64
    c = {f: rng.uniform(-0.1, 0.1, npt) for f in tp.inputs_c}
    if name != "enforce":
        c[0] = rng.uniform(-0.5, -0.3, npt)       # chi - 1
        c[17] = rng.uniform(-0.4, -0.2, npt)      # alpha - 1
    d = {s: rng.uniform(-0.2, 0.2, npt) for s in tp.inputs_d}
    rb = {f: rng.standard_normal(npt) for f in tp.outputs}
    dc = {f: rng.standard_normal(npt) for f in c}
    dd = {s: rng.standard_normal(npt) for s in d}
    cb, db = TP.vjp(tp, c, d, rb)
    lhs = sum(np.sum(cb.get(f, 0) * dc[f]) for f in c) + sum(np.sum(db.get(s, 0) * dd[s]) for s in d)
    h = 1e-6
    up = tp.evaluate({f: c[f] + h * dc[f] for f in c}, {s: d[s] + h * dd[s] for s in d})
    dn = tp.evaluate({f: c[f] - h * dc[f] for f in c}, {s: d[s] - h * dd[s] for s in d})
    rhs = sum(np.sum(rb[f] * (up[f] - dn[f]) / (2 * h)) for f in tp.outputs)
    assert abs(lhs - rhs) <= 1e-7 * abs(lhs), (lhs, rhs)


def test_tapes_are_the_current_kernels():
    """gen/trace_rhs.cpp, compiled from the kernels' point functions as they are
    now, records exactly the committed tapes, and the committed generated VJP
    header is what gen/emit.py makes of them: the adjoint differentiates the
    forward that runs."""
    import shutil
    import subprocess
    import tempfile
    gen = os.path.join(HERE, "..", "nr-amssncku_b200", "gen")
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "trace_rhs")
        subprocess.run([cxx, "-std=c++17", "-O0", "-o", exe, os.path.join(gen, "trace_rhs.cpp")], check=True)
        for mode in ("bssn", "z4c", "ham", "enforce"):
            out = subprocess.run([exe, mode], check=True, capture_output=True, text=True).stdout
            with open(os.path.join(gen, f"tape_{mode}.txt")) as fh:
                assert out == fh.read(), mode
    import emit
    with open(os.path.join(HERE, "..", "nr-amssncku_b200", "csrc", "rhs_vjp_gen.cuh")) as fh:
        assert emit.generate() == fh.read()
