"""GPU parity of the wave extraction (amss_engine_psi4, amss_engine_psi4_modes)
against the oracle (oracle/waves.py: getnp4 per block from the oracle's own
Christoffel symbols and Ricci tensor, the level's ghost sync, the level
interpolation and surf_Wave's quadrature).

Data: moving, spinning punctures (Lousto's data with momenta and spins, so
K_ij and its derivatives are not zero) plus seeded noise, on the three-level
test hierarchy; and an octant block (Symmetry 2) with a mirrored pair of
punctures, which exercises the mirrored stencils and the eight mirror images
of surf_Wave.  Bars: Psi4 within 1e-10 of the level's largest |Psi4| at every
point, modes within 1e-10 of the largest mode (relative max-norm)."""
import numpy as np
import pytest

import amss_b200
from amss_b200.hierarchy import box_in_box
import amr as OA
import interp as OI
import oracle as O
import waves as W

pytestmark = pytest.mark.gpu

MASSES = [0.5, 0.45]
POS = [[1.2, 0.3, -0.4], [-1.0, -0.2, 0.35]]
MOM = [[0.0, 0.1, 0.02], [0.01, -0.1, 0.0]]
SPIN = [[0.0, 0.02, 0.05], [0.01, 0.0, -0.04]]


def _state(H, noise=1e-6, seed=5):
    out = []
    for b in H.blocks:
        X, Y, Z = H.coords(b)
        st = O.get_lousto_nbhs(X, Y, Z, MASSES, POS, MOM, SPIN)
        gk, gj, gi = np.meshgrid(np.arange(b.ex[2]) + b.org[2], np.arange(b.ex[1]) + b.org[1],
                                 np.arange(b.ex[0]) + b.org[0], indexing="ij")
        for f in range(24):
            st[f] += noise * OA.grid_noise(b.level, f, gi, gj, gk, seed)
        out.append(st)
    return out


@pytest.fixture(scope="module")
def case():
    H = box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    init = _state(H)
    return H, init


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_psi4_matches_oracle_on_every_level(case, precision):
    H, init = case
    e = amss_b200.Engine.from_hierarchy(H, precision=precision, eps=0.1)
    try:
        for i, st in enumerate(init):
            e.set_state(i, st)
        states = {i: init[i] for i in range(len(H.blocks))}
        for lv in range(len(H.levels)):
            ref = W.psi4_level(H, lv, states, eps=0.1)
            e.psi4(lv)
            got = {bi: e.get_psi4(bi) for bi in ref}
            scale = max(np.abs(r).max() for r in ref.values())
            err = max(np.abs(got[bi] - ref[bi]).max() for bi in ref) / scale
            assert scale > 1e-6 and err <= 1e-10, (lv, err, scale)
    finally:
        e.close()


def test_psi4_modes_match_oracle(case):
    H, init = case
    e = amss_b200.Engine.from_hierarchy(H, eps=0.1)
    try:
        for i, st in enumerate(init):
            e.set_state(i, st)
        states = {i: init[i] for i in range(len(H.blocks))}
        for lv, rex in ((0, 6.0), (1, 2.0)):
            ref_psi = W.psi4_level(H, lv, states, eps=0.1)
            rp0, ip0 = W.extract(H, lv, ref_psi, rex, nquarter=4, maxl=4)
            e.psi4(lv)
            rp, ip = e.psi4_modes(lv, rex, nquarter=4, maxl=4)
            scale = max(np.abs(rp0).max(), np.abs(ip0).max())
            assert scale > 0
            assert np.abs(rp - rp0).max() <= 1e-10 * scale, (lv, np.abs(rp - rp0).max() / scale)
            assert np.abs(ip - ip0).max() <= 1e-10 * scale, (lv, np.abs(ip - ip0).max() / scale)
        # a sphere that leaves the level is refused
        with pytest.raises(amss_b200.AmssError):
            e.psi4_modes(1, 9.0, nquarter=4, maxl=4)
    finally:
        e.close()


def test_octant_modes_match_oracle():
    """Symmetry 2 on one block [0, 6]^3 (24 cells a side): mirrored stencils at
    the three symmetry planes and the eight mirror images of the sphere."""
    n, L = 24, 6.0
    X = O.cell_coords(0.0, L, n)
    bbox = [0.0, 0.0, 0.0, L, L, L]
    st = O.get_lousto_nbhs(X, X, X, [0.5, 0.5], [[1.5, 0.0, 0.0], [-1.5, 0.0, 0.0]],
                           [[0.0, 0.1, 0.0], [0.0, -0.1, 0.0]])
    _, _, gam, ric, _ = O.compute_rhs_bssn(X, X, X, st, symmetry=2, eps=0.1)
    rp_ref, ip_ref = W.getnp4(X, X, X, st, gam, ric, symmetry=2)
    e = amss_b200.Engine(symmetry=2, eps=0.1)
    try:
        b = e.add_block(0, (n, n, n), bbox, bbox)
        e.commit()
        e.set_state(b, st)
        e.psi4(0)
        got = e.get_psi4(b)
        scale = max(np.abs(rp_ref).max(), np.abs(ip_ref).max())
        assert _rel(got[0], rp_ref) * np.abs(rp_ref).max() <= 1e-10 * scale
        assert _rel(got[1], ip_ref) * np.abs(ip_ref).max() <= 1e-10 * scale
        rex = 3.0
        rp, ip = e.psi4_modes(0, rex, nquarter=4, maxl=4)
        patches = [(bbox, [n, n, n], 0, [(bbox, X, X, X, np.stack([rp_ref, ip_ref]))])]
        _, _, _, _, _, pts = W.sphere(4, 2)
        vals, found = OI.interp_points(patches, [(rex * a, rex * b_, rex * c) for a, b_, c in pts], [0, 1],
                                       [W.RPSI4_SOA, W.IPSI4_SOA], 2)
        assert all(found)
        rp0, ip0 = W.surf_wave(rex, vals, 4, 2, 4)
        ms = max(np.abs(rp0).max(), np.abs(ip0).max())
        assert np.abs(rp - np.array(rp0)).max() <= 1e-10 * ms
        assert np.abs(ip - np.array(ip0)).max() <= 1e-10 * ms
        # the ADM mass with the octant's factor 8 (the momenta are not integrated)
        comb = np.concatenate([W.admmass(X, X, X, st, symmetry=2), st[:14]])
        patches = [(bbox, [n, n, n], 0, [(bbox, X, X, X, comb)])]
        vals, _ = OI.interp_points(patches, [(rex * a, rex * b_, rex * c) for a, b_, c in pts], list(range(17)),
                                   W.MASS_SOA + [W.STATE_SOA[k] for k in range(14)], 2)
        ref = np.array(W.surf_masspang(rex, vals, 4, 2))
        got = e.adm_integrals(0, rex, nquarter=4)
        assert abs(got[0] - ref[0]) <= 1e-10 * abs(ref[0]) and np.all(got[1:] == 0.0)
    finally:
        e.close()


def test_adm_integrals_match_oracle(case):
    """surf_MassPAng: the mass integrand formed per block (not synchronised),
    17 values interpolated on the sphere, the sums; levels 0 and 1."""
    H, init = case
    e = amss_b200.Engine.from_hierarchy(H, eps=0.1)
    try:
        for i, st in enumerate(init):
            e.set_state(i, st)
        states = {i: init[i] for i in range(len(H.blocks))}
        for lv, rex in ((0, 6.0), (1, 2.0)):
            ref = np.array(W.adm_extract(H, lv, states, rex, nquarter=4))
            got = e.adm_integrals(lv, rex, nquarter=4)
            scale = np.abs(ref).max()
            assert np.abs(got - ref).max() <= 1e-10 * scale, (lv, got, ref)
        # the Psi4 fields survive the ADM integrand in the accumulator
        e.psi4(0)
        before = e.get_psi4(0)
        e.adm_integrals(0, 6.0, nquarter=4)
        assert np.array_equal(e.get_psi4(0), before)
    finally:
        e.close()


def test_z4c_engine_psi4_and_adm(case):
    """A Z4c run's analysis reads the first 24 fields (Z4c_class inherits
    Compute_Psi4 and AnalysisStuff); Theta does not enter."""
    H, init = case
    init25 = [np.concatenate([s, 1e-6 * np.ones((1,) + s.shape[1:])]) for s in init]
    e = amss_b200.Engine.from_hierarchy(H, eps=0.1, formulation="z4c")
    try:
        for i, st in enumerate(init25):
            e.set_state(i, st)
        states = {i: init[i] for i in range(len(H.blocks))}
        ref = W.psi4_level(H, 0, states, eps=0.1)
        e.psi4(0)
        scale = max(np.abs(r).max() for r in ref.values())
        assert max(np.abs(e.get_psi4(bi) - ref[bi]).max() for bi in ref) <= 1e-10 * scale
        adm = np.array(W.adm_extract(H, 0, states, 6.0, nquarter=4))
        assert np.abs(e.adm_integrals(0, 6.0, nquarter=4) - adm).max() <= 1e-10 * np.abs(adm).max()
    finally:
        e.close()
