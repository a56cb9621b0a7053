"""Known-answer checks of the CPU oracle (no GPU).

The reference ships no tests or golden vectors for this path, so the oracle is
pinned by analytic answers: Minkowski gives an exactly zero RHS; Brill-Lindquist
data at t = 0 has exactly zero chi, metric, lapse, shift and Gamma^i right-hand
sides without dissipation; its Hamiltonian constraint converges at 4th order;
the stencils are exact on polynomials of their order.
"""
import numpy as np
import pytest

import oracle as O

from helpers import generic_state


def test_minkowski_rhs_is_zero():
    X = O.cell_coords(-2.0, 2.0, 16)
    st = np.zeros((24, 16, 16, 16))
    gont, rhs, gam, ric, cons = O.compute_rhs_bssn(X, X, X, st, eps=0.1, co=0)
    assert gont == 0
    assert np.all(rhs == 0) and np.all(gam == 0) and np.all(ric == 0) and np.all(cons == 0)


def test_brill_lindquist_analytic_zeros():
    X, st, bbox, h = O.single_block_setup(24, -8.0, 8.0, 3, [1.0], [[0.1, 0.05, 0.02]])
    gont, rhs, *_ = O.compute_rhs_bssn(X, X, X, st, eps=0.0, co=1)
    assert gont == 0
    zero = ["chi", "gxx", "gxy", "gxz", "gyy", "gyz", "gzz", "Gamx", "Gamy", "Gamz", "Lap",
            "betax", "betay", "betaz", "dtSfx", "dtSfy", "dtSfz"]
    for name in zero:
        assert np.all(rhs[O.STATE_NAMES.index(name)] == 0), name
    for name in ["trK", "Axx", "Ayy", "Azz"]:
        assert np.abs(rhs[O.STATE_NAMES.index(name)]).max() > 1e-3, name


def _ham_far(n):
    X, st, bbox, h = O.single_block_setup(n, -8.0, 8.0, 3, [1.0], [[0.1, 0.05, 0.02]])
    _, _, _, _, cons = O.compute_rhs_bssn(X, X, X, st, eps=0.0, co=0)
    z, y, x = np.meshgrid(X, X, X, indexing="ij")
    r = np.sqrt((x - 0.1) ** 2 + (y - 0.05) ** 2 + (z - 0.02) ** 2)
    m = (r > 3) & (np.abs(x) < 6) & (np.abs(y) < 6) & (np.abs(z) < 6)
    return np.abs(cons[0][m]).max()


def test_hamiltonian_constraint_converges_at_fourth_order():
    ratio = _ham_far(32) / _ham_far(64)
    assert 12.0 < ratio < 20.0, ratio


def test_stencils_exact_on_polynomials():
    X = O.cell_coords(-1.0, 1.0, 14)
    Y = O.cell_coords(-1.5, 0.5, 12)
    Z = O.cell_coords(0.0, 2.0, 10)
    z, y, x = np.meshgrid(Z, Y, X, indexing="ij")
    f = x ** 4 + 2 * y ** 3 * x - z ** 4 + x * y * z + 0.5 * z ** 2 * y ** 2
    fx, fy, fz = O.fderivs(X, Y, Z, f)
    fxx, fxy, fxz, fyy, fyz, fzz = O.fdderivs(X, Y, Z, f)
    inner = (slice(2, -2), slice(2, -2), slice(2, -2))
    exact = {
        "fx": 4 * x ** 3 + 2 * y ** 3 + y * z, "fy": 6 * y ** 2 * x + x * z + z ** 2 * y,
        "fz": -4 * z ** 3 + x * y + z * y ** 2, "fxx": 12 * x ** 2, "fxy": 6 * y ** 2 + z,
        "fxz": y, "fyy": 12 * y * x + z ** 2, "fyz": x + 2 * z * y, "fzz": -12 * z ** 2 + y ** 2}
    got = {"fx": fx, "fy": fy, "fz": fz, "fxx": fxx, "fxy": fxy, "fxz": fxz, "fyy": fyy, "fyz": fyz, "fzz": fzz}
    for k in exact:
        err = np.abs(got[k][inner] - exact[k][inner]).max()
        assert err < 1e-9 * (1 + np.abs(exact[k][inner]).max()), (k, err)
    # the outermost planes are exactly zero (diff_new.f90:996-1002)
    for a in got.values():
        assert np.all(a[:, :, 0] == 0) and np.all(a[:, :, -1] == 0)
        assert np.all(a[:, 0, :] == 0) and np.all(a[0, :, :] == 0)


def test_enforce_ga_unit_determinant_and_trace_free():
    X = O.cell_coords(-1.0, 1.0, 10)
    st = generic_state(X, X, X)
    O.enforce_ga(st)
    g = np.array([[st[2] + 1, st[3], st[4]], [st[3], st[5] + 1, st[6]], [st[4], st[6], st[7] + 1]])
    a = np.array([[st[8], st[9], st[10]], [st[9], st[11], st[12]], [st[10], st[12], st[13]]])
    g = np.moveaxis(g, (0, 1), (-2, -1))
    a = np.moveaxis(a, (0, 1), (-2, -1))
    assert np.abs(np.linalg.det(g) - 1).max() < 1e-14
    tr = np.einsum("...ij,...ij->...", np.linalg.inv(g), a)
    assert np.abs(tr).max() < 1e-14


def test_rk4_on_linear_ode_is_fourth_order():
    # dy/dt = lam*y through the reference's low-storage RK4 (rungekutta4_rout.f90:94-139)
    lam = -0.7
    def run(dt, n):
        y0 = np.ones((2, 2, 2))
        for _ in range(n):
            K = lam * y0.copy()
            f1 = np.zeros_like(y0)
            O.rungekutta4_rout(dt, y0, f1, K, 0)
            for it in (1, 2, 3):
                k = lam * f1
                O.rungekutta4_rout(dt, y0, k, K, it)
                f1 = k
            y0 = f1.copy()
        return y0[0, 0, 0]
    e1 = abs(run(0.2, 5) - np.exp(lam))
    e2 = abs(run(0.1, 10) - np.exp(lam))
    assert 14 < e1 / e2 < 18


def test_nan_input_reported_outputs_untouched():
    X = O.cell_coords(-1.0, 1.0, 8)
    st = generic_state(X, X, X)
    st[5][3, 3, 3] = np.nan
    gont, rhs, *_ = O.compute_rhs_bssn(X, X, X, st, co=0)
    assert gont == 1 and np.all(rhs == 0)
    st = generic_state(X, X, X)
    st[22][3, 3, 3] = np.nan  # dtSfy is not among the checked fields (bssn_rhs.f90:110-113)
    gont, *_ = O.compute_rhs_bssn(X, X, X, st, co=0)
    assert gont == 0


def test_reflection_parity():
    """Mirroring the data through x = 0 maps every RHS onto itself with the
    field's x-parity (bssn_class.C:177-330), the reference's symmetry table."""
    X = O.cell_coords(-2.0, 2.0, 14)
    st = generic_state(X, X, X)
    par = O.BSSN_SOA[:, 0]
    st = 0.5 * (st + par[:, None, None, None] * st[:, :, :, ::-1])   # make the data x-symmetric
    _, rhs, *_ = O.compute_rhs_bssn(X, X, X, st, eps=0.1, co=1)
    mirrored = par[:, None, None, None] * rhs[:, :, :, ::-1]
    # the boundary planes are not mirror images in the reference itself: its
    # advection loop covers i = 1 but not i = ex (lopsidediff.f90:236-238)
    inner = (slice(None), slice(3, -3), slice(3, -3), slice(3, -3))
    assert np.abs(mirrored - rhs)[inner].max() <= 1e-12 * np.abs(rhs).max()
