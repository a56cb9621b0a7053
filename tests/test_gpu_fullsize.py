"""GPU parity at the sizes the bench times (CUDA path through the C ABI of
libamss_b200.so against the CPU oracle on the same inputs).

* single64 (one 64^3-interior block + 3 ghost cells on [-8, 8]^3,
  Brill-Lindquist m = 1 at (0.1, 0.05, 0.02), noise 1e-8): 100 FP64 RK4 steps
  replayed as a CUDA graph against 100 oracle steps, <= 1e-12 per field.
* amr (96^3 coarse on [-48, 48]^3 + 6 box-in-box levels around m = 0.5 at
  (+-3, 0, 0), 20 uneven blocks): one whole Berger-Oliger coarse step with the
  puncture tracking, graph replay against the oracle hierarchy, <= 1e-12 per
  field over all blocks (trK 5e-12: 112 fine steps of accumulated rounding on
  a small field), tracked positions equal to 1e-12.
* adjoint96 (96^3 interior on [-12, 12]^3, BL m = 1 at (0.1, 0.05, 0.02) +
  Gaussian on gamma~_xx): the gradient of sum H^2 dV after 40 FP64 steps with
  a checkpoint every 20 (two segments) against central differences (h = 1e-6)
  along a smooth gamma~_xx-field direction and a mass/position direction.

The oracle runs on the host cores (OpenMP); the amr case takes a few minutes.
"""
import numpy as np
import pytest

import amss_b200
import oracle as O
import amr as OA
from amss_b200 import initial
from amss_b200.hierarchy import box_in_box

from helpers import relerr

pytestmark = pytest.mark.gpu

POS1 = [[0.1, 0.05, 0.02]]


def test_single64_100_steps_graph():
    X, st0, bbox, h = O.single_block_setup(64, -8.0, 8.0, 3, [1.0], POS1, noise=1e-8, seed=1)
    dt = 0.25 * h
    n = len(X)
    e = amss_b200.Engine(precision="fp64", eps=0.1)
    b = e.add_block(0, (n, n, n), bbox, bbox)
    e.commit()
    e.set_state(b, st0)
    e.run_graph(0, dt, nsteps=1, replays=100)
    assert e.sync() == 0
    got = e.get_state(b)
    e.close()
    ref = st0.copy()
    for _ in range(100):
        O.bssn_step_single(X, X, X, bbox, ref, dt, eps=0.1)
    errs = [relerr(got[f], ref[f]) for f in range(24)]
    assert max(errs) <= 1e-12, errs


def test_amr_workload_one_coarse_step_with_tracking():
    pos = [[-3.0, 0.0, 0.0], [3.0, 0.0, 0.0]]
    H = box_in_box(96, 48.0, [tuple(p) for p in pos], 7, box_cells=48, seed=1, block_min=18, block_max=74)
    assert len(H.levels) == 7 and len(H.blocks) == 20
    init = OA.initial_state(H, [0.5, 0.5], pos, noise=0.0)
    dt0 = 0.25 * H.h0
    e = amss_b200.Engine.from_hierarchy(H, precision="fp64", eps=0.1)
    for i, st in enumerate(init):
        e.set_state(i, st)
    e.set_punctures(pos)
    e.run_coarse_graph(dt0, nsteps=1, replays=1)
    assert e.sync() == 0
    got = [e.get_state(i) for i in range(len(H.blocks))]
    got_pos = e.punctures()
    e.close()
    oh = OA.OracleHierarchy(H, eps=0.1)
    for i, st in enumerate(init):
        oh.set_state(i, st)
    oh.set_punctures(pos)
    assert oh.coarse_step(dt0) == 0
    ref = [oh.state(i) for i in range(len(H.blocks))]
    errs = np.zeros(24)
    for f in range(24):
        den = max(max(np.abs(r[f]).max() for r in ref), 1e-300)
        errs[f] = max(np.abs(g[f] - r[f]).max() for g, r in zip(got, ref)) / den
    # One coarse step is 112 RK4 steps of the finest levels, each an RHS
    # evaluation that agrees with the oracle's to rounding (<= 1e-12 per
    # evaluation, test_gpu_bssn_rhs.py); the rounding differences accumulate.
    # Measured: <= 3e-13 for every field but trK, 1.8e-12 for trK, whose
    # max-norm after one step is small against the O(1) terms its right-hand
    # side cancels.  The bar is 1e-12 for 23 fields and 5e-12 for trK.
    bar = np.full(24, 1e-12)
    bar[1] = 5e-12
    assert np.all(errs <= bar), errs
    # the positions follow the shift, which differs from the oracle's by the
    # rounding above: equal to 1e-12 (the y and z components stay ~1e-20)
    assert np.abs(np.asarray(got_pos) - np.asarray(oh.porg0)).max() <= 1e-12


def test_adjoint96_gradient_against_finite_differences():
    import torch
    from amss_b200.adjoint import Adjoint, BrillLindquist, hamiltonian_loss
    n, lo, hi = 96, -12.0, 12.0
    h = (hi - lo) / n
    X = O.cell_coords(lo - 3 * h, hi + 3 * h, n + 6)
    bbox = (lo - 3 * h,) * 3 + (hi + 3 * h,) * 3
    dt, nsteps, ck = 0.25 * h, 40, 20
    rng = np.random.default_rng(1)
    while True:
        c = rng.uniform(-4.0, 4.0, 3)
        if np.linalg.norm(c) < 4.0:
            break
    bump = initial.gaussian(X, X, X, 1e-4, 2.0, c)
    adj = Adjoint((len(X),) * 3, bbox)
    sel = torch.zeros(24, 1, 1, 1, dtype=torch.float64)
    sel[2] = 1.0

    def loss_of(m, p, gxx):
        st = BrillLindquist.apply(m, p, X, X, X) + sel * gxx[None]
        return hamiltonian_loss(st, adj, dt, nsteps, ck)

    m = torch.tensor([1.0], dtype=torch.float64, requires_grad=True)
    p = torch.tensor(POS1, dtype=torch.float64, requires_grad=True)
    gxx = torch.tensor(bump, requires_grad=True)
    L = loss_of(m, p, gxx)
    L.backward()
    gm, gp, gg = m.grad.numpy().copy(), p.grad.numpy().copy(), gxx.grad.numpy().copy()
    assert np.all(np.isfinite(gg))
    eps = 1e-6
    drng = np.random.default_rng(8)
    # the gamma~_xx field along a smooth seeded direction (a Gaussian of width 2
    # at a second random centre times a seeded plane wave) of amplitude 100, so
    # that h v is of the bump's own size (1e-4): L = 0.31 moves by only ~2e-3 h
    # per unit of this direction, and for h v ~ 1e-6 that change is below the
    # rounding L accumulates over 40 steps of 1e6 points (measured relative
    # error 1.9e-5 at h v = 1e-6, 8.9e-5 at 1e-7, 4e-8 at 1e-4: the 1/h
    # signature of rounding); then mass and position together
    z, y, x = np.meshgrid(X, X, X, indexing="ij")
    c2, k = drng.uniform(-3.0, 3.0, 3), drng.uniform(0.3, 0.8, 3)
    vfield = 100.0 * np.exp(-((x - c2[0]) ** 2 + (y - c2[1]) ** 2 + (z - c2[2]) ** 2) / 4.0) * \
        np.sin(k[0] * x + k[1] * y + k[2] * z)
    directions = [
        (np.zeros(1), np.zeros((1, 3)), vfield),
        (drng.standard_normal(1), drng.standard_normal((1, 3)), np.zeros(bump.shape)),
    ]
    with torch.no_grad():
        for trial, (vm, vp, vg) in enumerate(directions):
            an = float(np.dot(gm, vm) + np.sum(gp * vp) + np.sum(gg * vg))
            up = loss_of(m + eps * torch.tensor(vm), p + eps * torch.tensor(vp), gxx + eps * torch.tensor(vg))
            dn = loss_of(m - eps * torch.tensor(vm), p - eps * torch.tensor(vp), gxx - eps * torch.tensor(vg))
            fd = float(up - dn) / (2 * eps)
            assert abs(fd - an) <= 1e-6 * max(abs(fd), abs(an)), (trial, fd, an, float(L))
    adj.close()
