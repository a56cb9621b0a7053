"""Pins the point-interpolation oracle (oracle/interp.py: global_interp,
decide3d, polin3 / polint of fmisc.f90 and the patch / block search of
Parallel.C:5614-5667, MPatch.C:339-500) on the CPU: Neville's 6-point scheme
is exact on polynomials of degree <= 5 per axis, also through the mirrored
cells at a symmetry plane, and the search finds the finest covering level as
compute_Porg_rhs (bssn_class.C:6879-6932) walks down the levels."""
import numpy as np
import pytest

from amss_b200.hierarchy import box_in_box
import interp as OI


def _poly(x, y, z):
    return 1.0 + 0.3 * x - 0.2 * y ** 2 + 0.05 * x * y * z ** 2 + 0.01 * x ** 5 - 0.002 * z ** 4 * y


def _block(n, lo, h, zlo=None):
    zlo = lo if zlo is None else zlo
    X = lo + (np.arange(n) + 0.5) * h
    Z = zlo + (np.arange(n) + 0.5) * h
    z, y, x = np.meshgrid(Z, X, X, indexing="ij")
    return X, Z, (x, y, z)


def test_polint_exact_on_quintics():
    xa = [float(j) for j in range(6)]
    rng = np.random.default_rng(3)
    for _ in range(20):
        c = rng.uniform(-1, 1, 6)
        ya = [sum(c[p] * x ** p for p in range(6)) for x in xa]
        x = rng.uniform(0, 5)
        assert abs(OI.polint(xa, ya, x) - sum(c[p] * x ** p for p in range(6))) < 1e-12


def test_global_interp_exact_on_polynomial():
    X, Z, (x, y, z) = _block(16, -2.0, 0.25)
    f = _poly(x, y, z)
    rng = np.random.default_rng(5)
    for _ in range(25):
        p = rng.uniform(-1.9, 1.9, 3)
        got = OI.global_interp(f, X, X, Z, p[0], p[1], p[2], (1, 1, 1), 0)
        assert abs(got - _poly(*p)) < 1e-12 * max(1.0, abs(_poly(*p)))


@pytest.mark.parametrize("zpar", [1.0, -1.0])
def test_global_interp_mirrors_at_the_plane(zpar):
    """Symmetry 1: a block starting at z = 0; data even (parity +1) or odd
    (-1) in z; points within 2 cells of the plane use mirrored cells."""
    X, Z, (x, y, z) = _block(14, -1.75, 0.25, zlo=0.0)
    g = (lambda x, y, z: (1.0 + x * y) * (z ** 2 - 0.5 * z ** 4)) if zpar > 0 else \
        (lambda x, y, z: (1.0 + x - y ** 2) * (z - z ** 3))
    f = g(x, y, z)
    for p in [(0.1, -0.3, 0.05), (-0.7, 0.2, 0.2), (0.3, 0.3, 0.4)]:
        got = OI.global_interp(f, X, X, Z, p[0], p[1], p[2], (1, 1, zpar), 1)
        assert abs(got - g(*p)) < 1e-12


def test_search_walks_down_the_levels():
    H = box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    states = [np.zeros((24,) + tuple(b.ex[::-1])) for b in H.blocks]
    for i, b in enumerate(H.blocks):
        X, Y, Z = H.coords(b)
        z, y, x = np.meshgrid(Z, Y, X, indexing="ij")
        states[i][18] = _poly(x / 5, y / 5, z / 5)
    pts = [(1.2, 0.3, -0.4), (1.0, 0.1, -0.2), (6.0, -5.0, 2.0)]
    for p in pts:
        lev = len(H.levels) - 1
        while True:
            v, found = OI.interp_points(OI.hierarchy_patches(H, lev, states), [p], [18], [(1, 1, 1)])
            if found[0]:
                break
            lev -= 1
            assert lev >= 0
        assert abs(v[0][0] - _poly(p[0] / 5, p[1] / 5, p[2] / 5)) < 1e-12
        if p[0] > 5:
            assert lev == 0
        else:
            assert lev == len(H.levels) - 1


def test_oracle_tracking_follows_a_uniform_shift():
    """Brill-Lindquist data plus a uniform shift: over one coarse step (4
    steps of the finest level) the oracle's tracked puncture moves by minus
    the shift times the elapsed time (RK4 is exact for a constant right-hand
    side; the shift itself barely changes in that time)."""
    import amr as OA
    H = box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=0.0)
    beta = (0.05, -0.03, 0.02)
    for st in init:
        for v in range(3):
            st[18 + v] += beta[v]
    oh = OA.OracleHierarchy(H, eps=0.1)
    for i, st in enumerate(init):
        oh.set_state(i, st)
    oh.set_punctures([[1.2, 0.3, -0.4]])
    dt0 = 0.25 * H.h0
    assert oh.coarse_step(dt0) == 0
    moved = np.array(oh.porg0[0]) - np.array([1.2, 0.3, -0.4])
    assert np.abs(moved + dt0 * np.array(beta)).max() < 1e-5 * dt0
