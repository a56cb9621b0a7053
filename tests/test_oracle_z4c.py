"""Known-answer checks of the Z4c oracle (no GPU).

With Theta = 0 the Z4c right-hand side differs from the BSSN one only where
the formulation differs, and there by closed-form amounts: the trace of the
A~_ij source is taken from the Ricci scalar instead of the Hamiltonian
constraint, so A~_ij_rhs(Z4c) - A~_ij_rhs(BSSN) = -g~_ij alpha H / 3; Theta_rhs
= alpha H / 2 (+ advection and KO of Theta, zero here); trK_rhs is unchanged;
the Gamma^i damping term is the only other change.  H is the Hamiltonian
constraint the BSSN oracle returns.
"""
import numpy as np

import oracle as O

from helpers import generic_state

INNER = (slice(3, -3),) * 3


def _pair(seed=3, n=16, theta=None):
    X = O.cell_coords(-2.0, 2.0, n)
    st = generic_state(X, X, X, seed)
    tz = np.zeros((1,) + st.shape[1:]) if theta is None else theta[None]
    z = O.compute_rhs_z4c(X, X, X, np.concatenate([st, tz]), eps=0.1)
    b = O.compute_rhs_bssn(X, X, X, st, eps=0.1, co=0)
    return X, st, z, b


def test_minkowski_z4c_rhs_is_zero():
    X = O.cell_coords(-2.0, 2.0, 12)
    gont, rhs, gam, ric, cons = O.compute_rhs_z4c(X, X, X, np.zeros((25, 12, 12, 12)), eps=0.1)
    assert gont == 0
    assert np.all(rhs == 0) and np.all(gam == 0) and np.all(ric == 0) and np.all(cons == 0)


def test_z4c_with_zero_theta_matches_bssn_closed_forms():
    X, st, (gz, rz, gmz, riz, cz), (gb, rb, gmb, rib, cb) = _pair()
    assert gz == gb == 0
    same = ["chi", "trK", "gxy", "gxz", "gyz", "Lap", "betax", "betay", "betaz", "dtSfx", "dtSfy", "dtSfz"]
    for name in same:
        f = O.STATE_NAMES.index(name)
        assert np.array_equal(rz[f], rb[f]), name
    # KO of the diagonal metric acts on g = d + 1 in Z4c, on d in BSSN: round-off only
    for name in ["gxx", "gyy", "gzz"]:
        f = O.STATE_NAMES.index(name)
        assert np.abs(rz[f] - rb[f]).max() <= 1e-13 * np.abs(rb[f]).max(), name
    alpha = st[17] + 1.0
    H = cb[0]
    g = {"Axx": st[2] + 1, "Axy": st[3], "Axz": st[4], "Ayy": st[5] + 1, "Ayz": st[6], "Azz": st[7] + 1}
    for name, gij in g.items():
        f = O.STATE_NAMES.index(name)
        expect = -gij * alpha * H / 3.0
        err = np.abs(rz[f] - rb[f] - expect)[INNER].max()
        assert err <= 1e-12 * np.abs(rb[f]).max(), (name, err)
    assert np.allclose(rz[24][INNER], (0.5 * alpha * H)[INNER], rtol=1e-12, atol=1e-15)
    # diagnostic outputs (ricci_gamma + constraint_bssn) are the BSSN ones
    assert np.array_equal(gmz, gmb) and np.array_equal(riz, rib) and np.array_equal(cz, cb)


def test_theta_enters_through_trKd_and_damping():
    """A constant Theta = c shifts chi_rhs by (2/3) chi alpha 2c, trK_rhs by the
    damping kappa1 alpha c plus the change of (1/3) trKd^2, and Theta_rhs by the
    trKd^2 term of H minus the damping 2 kappa1 alpha c (no gradients of Theta)."""
    n = 16
    c = 1e-3
    X, st, z0, _ = _pair(n=n)
    _, _, z1, _ = _pair(n=n, theta=np.full((n, n, n), c))
    r0, r1 = z0[1], z1[1]
    chin1, alpha, K = st[0] + 1, st[17] + 1, st[1]
    k1 = 0.02
    d_chi = (2.0 / 3.0) * chin1 * alpha * (2 * c)
    assert np.allclose((r1[0] - r0[0])[INNER], d_chi[INNER], rtol=1e-9, atol=1e-14)
    d_trk = alpha * ((K + 2 * c) ** 2 - K ** 2) / 3.0 + alpha * k1 * c
    assert np.allclose((r1[1] - r0[1])[INNER], d_trk[INNER], rtol=1e-9, atol=1e-14)
    d_tz = alpha * (2.0 / 3.0) * ((K + 2 * c) ** 2 - K ** 2) / 2.0 - alpha * 2 * k1 * c
    assert np.allclose((r1[24] - r0[24])[INNER], d_tz[INNER], rtol=1e-9, atol=1e-14)


def test_z4c_nan_check_covers_theta():
    X = O.cell_coords(-2.0, 2.0, 10)
    st = np.zeros((25, 10, 10, 10))
    st[24, 4, 4, 4] = np.nan
    gont, rhs, *_ = O.compute_rhs_z4c(X, X, X, st, eps=0.1)
    assert gont == 1 and np.all(rhs == 0)
