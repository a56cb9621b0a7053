"""GPU parity of the fused, batched RK4 step (engine) against the oracle's
single-block level-0 step (enforce_ga, compute_rhs_bssn, sommerfeld_routbam,
rungekutta4_rout, lowerboundset per substep, bssn_class.C:2981-3915).

The engine applies enforce_ga to what a substep writes, so its state after a
step is enforce_ga of the reference's; the comparison applies enforce_ga to
the oracle's result.  FP64 bar 1e-12; mixed-precision bar 1e-6 (relative
max-norm per field)."""
import numpy as np
import pytest

import oracle as O
import amss_b200

from helpers import generic_state, relerr

pytestmark = pytest.mark.gpu


def _run(precision, st0, X, bbox, dt, nsteps, eps=0.1):
    n = len(X)
    e = amss_b200.Engine(precision=precision, eps=eps)
    b = e.add_block(0, (n, n, n), bbox, bbox)
    e.commit()
    e.set_state(b, st0)
    e.enforce()
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
    O.enforce_ga(st)
    return st


@pytest.mark.parametrize("case", ["bl", "generic"])
def test_fp64_step_matches_oracle(case):
    if case == "bl":
        X, st0, bbox, h = O.single_block_setup(24, -6.0, 6.0, 3, [1.0], [[0.1, 0.05, 0.02]], noise=1e-8)
    else:
        X = O.cell_coords(-3.0, 3.0, 22)
        h = X[1] - X[0]
        bbox = (-3.0, -3.0, -3.0, 3.0, 3.0, 3.0)
        st0 = generic_state(X, X, X, seed=12, amp=0.5)
    dt = 0.25 * h
    ref = _oracle(st0, X, bbox, dt, 3)
    got = _run("fp64", st0, X, bbox, dt, 3)
    errs = [relerr(got[f], ref[f]) for f in range(24)]
    assert max(errs) <= 1e-12, errs


def test_mixed_step_error_bound():
    X, st0, bbox, h = O.single_block_setup(24, -6.0, 6.0, 3, [1.0], [[0.1, 0.05, 0.02]], noise=1e-8)
    dt = 0.25 * h
    ref = _oracle(st0, X, bbox, dt, 3)
    got = _run("mixed", st0, X, bbox, dt, 3)
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
    e.enforce()
    e.run_graph(0, dt, nsteps=2, replays=2)
    assert e.sync() == 0
    assert np.array_equal(e.get_state(b), eager)
    assert e.launches == 1 + 4 * 4
