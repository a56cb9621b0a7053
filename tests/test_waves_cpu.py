"""The wave-extraction oracle (oracle/waves.py, oracle/psi4_oracle.c) against
known answers, without a GPU.

* getnp4 of flat space is exactly 0.
* Around one Brill-Lindquist puncture at the origin the spatial tetrad
  (radial v, azimuthal u, polar w, Gram-Schmidt in the physical metric) sees a
  spherically symmetric tidal field, E(u, u) = E(w, w), E(u, w) = 0, so Psi4
  vanishes up to truncation error: it is a small fraction of the electric
  field's size and falls at 4th order when the grid is refined.
* surf_Wave's basis sqrt((2l+1)/4pi) d^l_{m,2}(theta) e^{i m phi} is
  orthonormal under its quadrature (Gauss-Legendre in cos(theta), midpoints
  in phi): a field made of known modes gives back rex times each coefficient.
* The Gauss-Legendre nodes and weights and the Wigner d function agree with
  closed forms.
"""
import math

import numpy as np
import pytest

import oracle as O
import waves as W


def _block(n, lo, hi):
    X = O.cell_coords(lo, hi, n)
    return X, X.copy(), X.copy()


def test_flat_space_has_no_psi4():
    X, Y, Z = _block(16, -4.0, 4.0)
    st = np.zeros((24, 16, 16, 16))
    _, _, gam, ric, _ = O.compute_rhs_bssn(X, Y, Z, st)
    rp, ip = W.getnp4(X, Y, Z, st, gam, ric)
    assert np.all(rp == 0.0) and np.all(ip == 0.0)


def _bl_psi4(n):
    X, Y, Z = _block(n, -6.0, 6.0)
    st = O.get_lousto_nbhs(X, Y, Z, [1.0], [[0.0, 0.0, 0.0]])
    _, _, gam, ric, _ = O.compute_rhs_bssn(X, Y, Z, st)
    rp, ip = W.getnp4(X, Y, Z, st, gam, ric)
    zz, yy, xx = np.meshgrid(Z, Y, X, indexing="ij")
    r = np.sqrt(xx * xx + yy * yy + zz * zz)
    # the shell 3 <= r <= 4.5, away from the puncture and from the block's faces
    sel = (r >= 3.0) & (r <= 4.5)
    return np.abs(rp[sel]).max(), np.abs(ip[sel]).max(), np.abs(ric[0][sel]).max()


def test_single_puncture_psi4_vanishes_at_fourth_order():
    r1, i1, e1 = _bl_psi4(48)
    r2, i2, e2 = _bl_psi4(96)
    assert r1 < 1e-2 * e1 and i1 < 1e-2 * e1
    # halving h cuts the truncation error by ~16
    assert r2 < r1 / 8 and i2 < i1 / 8


def test_gauss_legendre_and_wigner_d_closed_forms():
    x, w = W.gaulegf(-1.0, 1.0, 12)
    for k in range(0, 24):
        exact = 0.0 if k % 2 else 2.0 / (k + 1)
        assert abs(sum(wi * xi ** k for xi, wi in zip(x, w)) - exact) < 1e-14
    for th in (0.1, 0.9, 2.0, 3.0):
        c = math.cos(th)
        assert abs(W.wigner_d(2, 2, 2, c) - math.cos(th / 2) ** 4) < 1e-15
        assert abs(W.wigner_d(2, -2, 2, c) - math.sin(th / 2) ** 4) < 1e-15
        assert abs(W.wigner_d(2, 0, 2, c) - math.sqrt(6) / 4 * math.sin(th) ** 2) < 1e-15
        assert abs(W.wigner_d(2, 1, 2, c) - math.sin(th) / 2 * (1 + c)) < 1e-15


@pytest.mark.parametrize("nquarter", [6, 10])
def test_surf_wave_recovers_known_modes(nquarter):
    maxl, rex = 4, 7.5
    rng = np.random.default_rng(3)
    modes = [(l, m) for l in range(2, maxl + 1) for m in range(-l, l + 1)]
    coef = {lm: complex(rng.standard_normal(), rng.standard_normal()) for lm in modes}
    ct, wt, n_theta, n_phi, dphi, pts = W.sphere(nquarter, 0)
    vals = []
    for n, (a, b, c) in enumerate(pts):
        i, j = divmod(n, n_phi)
        ph = (j + 0.5) * dphi
        z = sum(coef[(l, m)] * math.sqrt((2 * l + 1) / 4 / math.pi) * W.wigner_d(l, m, 2, ct[i]) *
                complex(math.cos(m * ph), math.sin(m * ph)) for l, m in modes)
        vals.append((z.real, z.imag))
    rp, ip = W.surf_wave(rex, vals, nquarter, 0, maxl)
    for k, lm in enumerate(modes):
        assert abs(rp[k] - rex * coef[lm].real) < 1e-12 * rex
        assert abs(ip[k] - rex * coef[lm].imag) < 1e-12 * rex


def _adm_single_block(masses, pos, mom=None, spin=None, rex=3.0, n=48, L=6.0, nquarter=8):
    import interp as OI
    X = O.cell_coords(-L, L, n)
    st = O.get_lousto_nbhs(X, X, X, masses, pos, mom, spin)
    comb = np.concatenate([W.admmass(X, X, X, st), st[:14]])
    bb = [-L] * 3 + [L] * 3
    patches = [(bb, [n] * 3, 0, [(bb, X, X, X, comb)])]
    _, _, _, _, _, pts = W.sphere(nquarter, 0)
    vals, found = OI.interp_points(patches, [(rex * a, rex * b, rex * c) for a, b, c in pts], list(range(17)),
                                   W.MASS_SOA + [W.STATE_SOA[k] for k in range(14)], 0)
    assert all(found)
    return W.surf_masspang(rex, vals, nquarter, 0)


def test_adm_mass_of_a_puncture():
    """Brill-Lindquist: the mass integrand is -d_i psi / (2 pi), and psi is
    harmonic, so the sphere gives the bare mass at any radius."""
    out = _adm_single_block([1.0], [[0.0, 0.0, 0.0]])
    assert abs(out[0] - 1.0) < 1e-4
    assert max(abs(v) for v in out[1:]) < 1e-12


def test_adm_momentum_and_spin_of_a_boosted_spinning_puncture():
    """Bowen-York momentum and spin: the reference's integrand carries psi^6
    K_ij = psi^4 A^_ij, so at radius r the momentum reads P (1 + M/2r)^4, and
    the spin S (to the accuracy of the approximate data)."""
    P, S, r = 0.1, 0.2, 3.0
    out = _adm_single_block([1.0], [[0.0, 0.0, 0.0]], [[P, 0.0, 0.0]], [[0.0, 0.0, S]], rex=r)
    assert abs(out[1] / (P * (1 + 1.0 / (2 * r)) ** 4) - 1) < 0.05
    assert abs(out[6] / S - 1) < 0.05
    assert max(abs(out[2]), abs(out[3]), abs(out[4]), abs(out[5])) < 1e-3 * P
