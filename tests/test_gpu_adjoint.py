"""GPU tests of the adjoint path: puncture initial data (get_lousto_nbhs_) and
its mass / position VJP, the FP64 forward of amss_adjoint_* against the
oracle's level-0 step and Hamiltonian constraint, and the reverse sweep
against central finite differences (h = 1e-6) of the same forward along
seeded random directions -- in the full initial state, and, through the two
torch.autograd.Functions, in (mass, position, gamma~_xx field) as the
96^3 adjoint workload does at a size the test finishes in seconds.

Tolerances: the forward 1e-12 relative (max-norm per field) against the
oracle; the loss 1e-10 relative; directional derivatives 1e-6 relative to
the largest of |<grad, v>| and |FD| (the FD of an O(1e-3) loss with
h = 1e-6 carries roughly 1e-9 of rounding)."""
import numpy as np
import pytest

import oracle as O
import amss_b200
from amss_b200 import dropin, initial

from helpers import relerr

pytestmark = pytest.mark.gpu

POS = [[0.1, 0.05, 0.02]]


def _loss_oracle(X, st, bbox, gw=3):
    """sum over cells gw from every face of H^2 dV, H from the oracle's
    constraint output (compute_rhs_bssn with co = 0)."""
    H = O.compute_rhs_bssn(X, X, X, st, eps=0.1, co=0)[4][0]
    h = X[1] - X[0]
    return float(np.sum(H[gw:-gw, gw:-gw, gw:-gw] ** 2) * h ** 3)


@pytest.mark.parametrize("spinning", [False, True])
def test_lousto_matches_oracle(spinning):
    X = O.cell_coords(-3.0, 3.5, 26)
    Y = O.cell_coords(-2.5, 2.0, 18)
    Z = O.cell_coords(-1.5, 3.0, 20)
    m = [0.6, 0.4]
    pos = [[0.1, 0.05, 0.02], [-1.0, 0.5, X[7]]]
    mom = [[0.1, -0.2, 0.05], [0.0, 0.3, 0.0]] if spinning else None
    spin = [[0.0, 0.1, 0.2], [0.05, 0.0, -0.1]] if spinning else None
    got = dropin.get_lousto_nbhs(X, Y, Z, m, pos, mom, spin)
    ref = O.get_lousto_nbhs(X, Y, Z, m, pos, mom, spin)
    for f in range(24):
        assert relerr(got[f], ref[f]) <= 1e-13, f


def test_lousto_on_a_cell_centre():
    """A puncture exactly on a cell centre takes r = dx/2 there
    (initial_puncture.f90:2022)."""
    X = O.cell_coords(-2.0, 2.0, 16)
    pos = [[X[8], X[5], X[9]]]
    got = dropin.get_lousto_nbhs(X, X, X, [1.0], pos)
    ref = O.get_lousto_nbhs(X, X, X, [1.0], pos)
    assert np.all(np.isfinite(got))
    for f in range(24):
        assert relerr(got[f], ref[f]) <= 1e-13, f


def test_lousto_vjp_matches_finite_differences():
    X = O.cell_coords(-3.0, 3.0, 20)
    m = np.array([0.6, 0.4])
    pos = np.array([[0.4, 0.05, 0.02], [-0.9, 0.1, -0.2]])
    rng = np.random.default_rng(4)
    sb = rng.standard_normal((24, 20, 20, 20))
    dm, dp = dropin.lousto_vjp(X, X, X, m, pos, sb)
    h = 1e-6
    for trial in range(4):
        vm = rng.standard_normal(2)
        vp = rng.standard_normal((2, 3))
        up = O.get_lousto_nbhs(X, X, X, m + h * vm, pos + h * vp)
        dn = O.get_lousto_nbhs(X, X, X, m - h * vm, pos - h * vp)
        fd = np.sum(sb * (up - dn)) / (2 * h)
        an = np.dot(dm, vm) + np.sum(dp * vp)
        assert abs(fd - an) <= 1e-6 * max(abs(fd), abs(an)), (trial, fd, an)


def test_initial_state_matches_oracle():
    """The product's hierarchy initial data equals the oracle's to rounding
    (the inputs the tests compare on are the inputs the bench runs)."""
    import amr as OA
    from amss_b200.hierarchy import box_in_box
    H = box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    got = initial.initial_state(H, [0.6, 0.4], [[1.2, 0.3, -0.4], [-2, 0, 0]], noise=1e-6, seed=1, nf=25)
    ref = OA.initial_state(H, [0.6, 0.4], [[1.2, 0.3, -0.4], [-2, 0, 0]], noise=1e-6, seed=1, nf=25)
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert g.shape == r.shape
        assert np.max(np.abs(g - r)) <= 1e-14 * max(1.0, np.max(np.abs(r)))


def _block(n=20, lo=-2.5, hi=2.5, noise=1e-8):
    X, st0, bbox, h = O.single_block_setup(n, lo, hi, 3, [1.0], POS, noise=noise)
    return X, st0, bbox, h


def test_forward_matches_oracle_and_loss():
    X, st0, bbox, h = _block()
    dt = 0.25 * h
    adj = amss_b200.adjoint.Adjoint((len(X),) * 3, bbox)
    adj.set_state(st0)
    loss = adj.forward(dt, 5, 2)
    got = adj.get_state()
    ref = st0.copy()
    for _ in range(5):
        O.bssn_step_single(X, X, X, bbox, ref, dt, eps=0.1)
    errs = [relerr(got[f], ref[f]) for f in range(24)]
    assert max(errs) <= 1e-12, errs
    lref = _loss_oracle(X, ref, bbox)
    assert abs(loss - lref) <= 1e-10 * lref, (loss, lref)
    adj.close()


def _directional(adj, st0, dt, nsteps, ck, v, h=1e-6):
    adj.set_state(st0 + h * v)
    up = adj.forward(dt, nsteps, ck)
    adj.set_state(st0 - h * v)
    dn = adj.forward(dt, nsteps, ck)
    return (up - dn) / (2 * h)


def test_gradient_matches_finite_differences_full_state():
    """Eight seeded directions in the full initial state.  The shift components
    are left out of the directions: at t = 0 they sit at the noise level, where
    a 1e-6 step would flip the upwind side of the advection stencil, a kink the
    finite difference straddles.  chi and the lapse are perturbed relative to
    their value: near the puncture chi ~ 1e-3, and an absolute 1e-6 step there
    leaves an O((1e-3)^2) truncation error in the central difference."""
    X, st0, bbox, h = _block(noise=1e-6)
    dt = 0.25 * h
    nsteps, ck = 6, 4
    adj = amss_b200.adjoint.Adjoint((len(X),) * 3, bbox)
    adj.set_state(st0)
    adj.forward(dt, nsteps, ck)
    g = adj.backward()
    assert np.all(np.isfinite(g))
    rng = np.random.default_rng(11)
    for trial in range(8):
        v = rng.standard_normal(st0.shape)
        v[18:21] = 0.0
        v *= np.abs(st0).max(axis=(1, 2, 3), keepdims=True).clip(1e-3, 1.0)
        v[0] = rng.standard_normal(st0.shape[1:]) * (1.0 + st0[0])
        v[17] = rng.standard_normal(st0.shape[1:]) * (1.0 + st0[17])
        an = float(np.sum(g * v))
        fd = _directional(adj, st0, dt, nsteps, ck, v)
        assert abs(fd - an) <= 1e-6 * max(abs(fd), abs(an)), (trial, fd, an)
    adj.close()


def test_gradient_with_shift_directions():
    """Directions that perturb the shift too.  The state carries a smooth
    shift bounded away from zero (|beta^i| >= 0.02), so a 1e-6 step keeps the
    upwind side of every advection stencil and the central difference sees
    no kink; the directions then include beta^i, B^i and every other field."""
    X, st0, bbox, h = _block(noise=1e-6)
    z, y, x = np.meshgrid(X, X, X, indexing="ij")
    st0[18] += 0.05 + 0.02 * np.sin(0.7 * x) * np.cos(0.5 * y)
    st0[19] += -0.04 + 0.015 * np.cos(0.6 * z)
    st0[20] += 0.03 + 0.008 * np.sin(0.4 * x + 0.3 * z)
    assert np.abs(st0[18:21]).min() >= 0.02
    dt = 0.25 * h
    nsteps, ck = 6, 4
    adj = amss_b200.adjoint.Adjoint((len(X),) * 3, bbox)
    adj.set_state(st0)
    adj.forward(dt, nsteps, ck)
    g = adj.backward()
    assert np.all(np.isfinite(g))
    rng = np.random.default_rng(13)
    for trial in range(4):
        v = rng.standard_normal(st0.shape)
        v *= np.abs(st0).max(axis=(1, 2, 3), keepdims=True).clip(1e-3, 1.0)
        v[0] = rng.standard_normal(st0.shape[1:]) * (1.0 + st0[0])
        v[17] = rng.standard_normal(st0.shape[1:]) * (1.0 + st0[17])
        an = float(np.sum(g * v))
        fd = _directional(adj, st0, dt, nsteps, ck, v)
        assert abs(fd - an) <= 1e-6 * max(abs(fd), abs(an)), (trial, fd, an)
    adj.close()


def test_checkpoint_interval_does_not_change_the_gradient():
    X, st0, bbox, h = _block(n=16, lo=-2.0, hi=2.0)
    dt = 0.25 * h
    grads = []
    for ck in (1, 3, 7):
        adj = amss_b200.adjoint.Adjoint((len(X),) * 3, bbox)
        adj.set_state(st0)
        adj.forward(dt, 7, ck)
        grads.append(adj.backward())
        adj.close()
    for g in grads[1:]:
        for f in range(24):
            assert relerr(g[f], grads[0][f]) <= 1e-12, f


def test_autograd_mass_position_gxx_against_finite_differences():
    """The adjoint workload's gradient (mass, 3 position components, full
    gamma~_xx field with a Gaussian bump) at a reduced size: 20^3 interior on
    [-2.5, 2.5]^3, 6 steps, checkpoint every 4."""
    import torch
    from amss_b200.adjoint import Adjoint, BrillLindquist, hamiltonian_loss
    n, lo, hi = 20, -2.5, 2.5
    h = (hi - lo) / n
    a_lo, a_hi = lo - 3 * h, hi + 3 * h
    X = O.cell_coords(a_lo, a_hi, n + 6)
    bbox = (a_lo,) * 3 + (a_hi,) * 3
    dt, nsteps, ck = 0.25 * h, 6, 4
    rng = np.random.default_rng(5)
    c = rng.uniform(-1, 1, 3)
    c = 1.0 * c / max(np.linalg.norm(c), 1.0)
    bump = initial.gaussian(X, X, X, 1e-4, 0.5, c)
    adj = Adjoint((len(X),) * 3, bbox)
    sel = torch.zeros(24, 1, 1, 1, dtype=torch.float64)
    sel[2] = 1.0

    def loss_of(m, pos, gxx):
        st = BrillLindquist.apply(m, pos, X, X, X) + sel * gxx[None]
        return hamiltonian_loss(st, adj, dt, nsteps, ck)

    m = torch.tensor([1.0], dtype=torch.float64, requires_grad=True)
    pos = torch.tensor(POS, dtype=torch.float64, requires_grad=True)
    gxx = torch.tensor(bump, requires_grad=True)
    L = loss_of(m, pos, gxx)
    L.backward()
    grads = (m.grad.numpy().copy(), pos.grad.numpy().copy(), gxx.grad.numpy().copy())
    eps = 1e-6
    with torch.no_grad():
        for trial in range(8):
            vm = rng.standard_normal(1)
            vp = rng.standard_normal((1, 3))
            vg = rng.standard_normal(bump.shape) * 1e-2
            an = float(np.dot(grads[0], vm) + np.sum(grads[1] * vp) + np.sum(grads[2] * vg))
            up = loss_of(m + eps * torch.tensor(vm), pos + eps * torch.tensor(vp), gxx + eps * torch.tensor(vg))
            dn = loss_of(m - eps * torch.tensor(vm), pos - eps * torch.tensor(vp), gxx - eps * torch.tensor(vg))
            fd = float(up - dn) / (2 * eps)
            assert abs(fd - an) <= 1e-6 * max(abs(fd), abs(an)), (trial, fd, an)
    adj.close()


def test_gradient_matches_finite_differences_of_the_oracle_forward():
    """The gradient against central differences (h = 1e-6) of the plain FP64
    forward of the oracle (its level-0 step, bssn_class.C:2981-3700 restated,
    and its constraint output), not of the GPU forward: 14^3 interior, 3 steps,
    checkpoint every 2, two seeded directions."""
    X, st0, bbox, h = _block(n=14, lo=-1.75, hi=1.75, noise=1e-6)
    dt, nsteps, ck = 0.25 * h, 3, 2

    def oracle_loss(st):
        st = st.copy()
        for _ in range(nsteps):
            O.bssn_step_single(X, X, X, bbox, st, dt, eps=0.1)
        return _loss_oracle(X, st, bbox)

    adj = amss_b200.adjoint.Adjoint((len(X),) * 3, bbox)
    adj.set_state(st0)
    loss = adj.forward(dt, nsteps, ck)
    g = adj.backward()
    adj.close()
    assert abs(loss - oracle_loss(st0)) <= 1e-10 * loss
    rng = np.random.default_rng(21)
    for trial in range(2):
        v = rng.standard_normal(st0.shape)
        v[18:21] = 0.0
        v *= np.abs(st0).max(axis=(1, 2, 3), keepdims=True).clip(1e-3, 1.0)
        v[0] = rng.standard_normal(st0.shape[1:]) * (1.0 + st0[0])
        v[17] = rng.standard_normal(st0.shape[1:]) * (1.0 + st0[17])
        an = float(np.sum(g * v))
        fd = (oracle_loss(st0 + 1e-6 * v) - oracle_loss(st0 - 1e-6 * v)) / 2e-6
        assert abs(fd - an) <= 1e-6 * max(abs(fd), abs(an)), (trial, fd, an)
