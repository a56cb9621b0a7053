"""GPU parity of the fused, batched RK4 step (engine) against the oracle's
single-block level-0 step (enforce_ga, compute_rhs_bssn, sommerfeld_routbam,
rungekutta4_rout, lowerboundset per substep, bssn_class.C:2981-3915).

The engine's state after a step equals the reference's (enforce_ga runs in
place on U0 at the start of each step, as bssn_class.C:3052 does).  FP64 bar
1e-12; mixed-precision bar 1e-6 (relative max-norm per field)."""
import numpy as np
import pytest

import oracle as O
import amss_b200

from helpers import generic_state, relerr

pytestmark = pytest.mark.gpu


def _run(precision, st0, X, bbox, dt, nsteps, eps=0.1, kernel="split"):
    n = len(X)
    e = amss_b200.Engine(precision=precision, eps=eps, kernel=kernel)
    b = e.add_block(0, (n, n, n), bbox, bbox)
    e.commit()
    e.set_state(b, st0)
    for _ in range(nsteps):
        e.step(0, dt)
    assert e.sync() == 0
    out = e.get_state(b)
    e.close()
    return out


def _oracle(st0, X, bbox, dt, nsteps, eps=0.1):
    st = st0.copy()
    for _ in range(nsteps):
        O.bssn_step_single(X, X, X, bbox, st, dt, eps=eps)
    return st


@pytest.mark.parametrize("kernel", ["split", "fused"])
@pytest.mark.parametrize("case", ["bl", "generic"])
def test_fp64_step_matches_oracle(case, kernel):
    if case == "bl":
        X, st0, bbox, h = O.single_block_setup(24, -6.0, 6.0, 3, [1.0], [[0.1, 0.05, 0.02]], noise=1e-8)
    else:
        X = O.cell_coords(-3.0, 3.0, 22)
        h = X[1] - X[0]
        bbox = (-3.0, -3.0, -3.0, 3.0, 3.0, 3.0)
        st0 = generic_state(X, X, X, seed=12, amp=0.5)
    dt = 0.25 * h
    ref = _oracle(st0, X, bbox, dt, 3)
    got = _run("fp64", st0, X, bbox, dt, 3, kernel=kernel)
    errs = [relerr(got[f], ref[f]) for f in range(24)]
    assert max(errs) <= 1e-12, errs


@pytest.mark.parametrize("kernel", ["split", "fused"])
def test_mixed_step_error_bound(kernel):
    X, st0, bbox, h = O.single_block_setup(24, -6.0, 6.0, 3, [1.0], [[0.1, 0.05, 0.02]], noise=1e-8)
    dt = 0.25 * h
    ref = _oracle(st0, X, bbox, dt, 3)
    got = _run("mixed", st0, X, bbox, dt, 3, kernel=kernel)
    errs = [relerr(got[f], ref[f]) for f in range(24)]
    assert max(errs) <= 1e-6, errs


def test_graph_replay_equals_eager():
    X, st0, bbox, h = O.single_block_setup(16, -4.0, 4.0, 3, [1.0], [[0.1, 0.05, 0.02]], noise=1e-8)
    dt = 0.25 * h
    eager = _run("fp64", st0, X, bbox, dt, 4)
    n = len(X)
    e = amss_b200.Engine(precision="fp64")
    b = e.add_block(0, (n, n, n), bbox, bbox)
    e.commit()
    e.set_state(b, st0)
    e.run_graph(0, dt, nsteps=2, replays=2)
    assert e.sync() == 0
    assert np.array_equal(e.get_state(b), eager)
    # per step: enforce pass, 4 x (stencil pass + pointwise pass + face pass), ring rotation
    assert e.launches == 4 * 14
