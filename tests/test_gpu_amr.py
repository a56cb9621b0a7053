"""GPU parity of the batched Berger-Oliger evolution (engine: per-level fused
substeps, same-level ghost sync, restrict3 / prolong3 with time
interpolation, CUDA graph of a coarse step) against the CPU oracle hierarchy
(oracle/amr.py), on a small three-level box-in-box hierarchy of uneven
blocks.  FP64 bar 1e-12, mixed bar 1e-6 (relative max-norm per field over all
blocks of all levels)."""
import numpy as np
import pytest

import amss_b200
from amss_b200.hierarchy import box_in_box
import amr as OA

pytestmark = pytest.mark.gpu


def small_hierarchy():
    return box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)


def _run_oracle(H, init, dt0, steps):
    oh = OA.OracleHierarchy(H, eps=0.1)
    for i, st in enumerate(init):
        oh.set_state(i, st)
    for _ in range(steps):
        assert oh.coarse_step(dt0) == 0
    return [oh.state(i).copy() for i in range(len(H.blocks))]


def _run_engine(H, init, dt0, steps, precision="fp64", graph=False, kernel="split"):
    e = amss_b200.Engine.from_hierarchy(H, precision=precision, eps=0.1, kernel=kernel)
    for i, st in enumerate(init):
        e.set_state(i, st)
    if graph:
        e.run_coarse_graph(dt0, nsteps=1, replays=steps)
    else:
        for _ in range(steps):
            e.coarse_step(dt0)
    assert e.sync() == 0
    out = [e.get_state(i) for i in range(len(H.blocks))]
    e.close()
    return out


def _errs(got, ref):
    errs = np.zeros(24)
    for f in range(24):
        den = max(max(np.abs(r[f]).max() for r in ref), 1e-300)
        errs[f] = max(np.abs(g[f] - r[f]).max() for g, r in zip(got, ref)) / den
    return errs


def test_hierarchy_shape():
    H = small_hierarchy()
    assert len(H.levels) == 3
    assert all(len(p.blocks) >= 2 for lv in H.levels for p in lv)
    assert len({H.blocks[i].ex for i in range(len(H.blocks))}) > 3   # uneven blocks


@pytest.fixture(scope="module")
def fp64_reference():
    H = small_hierarchy()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-8)
    dt0 = 0.25 * H.h0
    return H, init, dt0, _run_oracle(H, init, dt0, 2)


@pytest.mark.parametrize("kernel", ["split", "fused"])
def test_fp64_amr_matches_oracle(fp64_reference, kernel):
    H, init, dt0, ref = fp64_reference
    got = _run_engine(H, init, dt0, 2, kernel=kernel)
    errs = _errs(got, ref)
    assert errs.max() <= 1e-12, errs


def test_graph_coarse_step_equals_eager():
    H = small_hierarchy()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-8)
    dt0 = 0.25 * H.h0
    a = _run_engine(H, init, dt0, 3)
    b = _run_engine(H, init, dt0, 3, graph=True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_mixed_amr_error_bound(fp64_reference):
    H, init, dt0, ref = fp64_reference
    got = _run_engine(H, init, dt0, 2, precision="mixed")
    errs = _errs(got, ref)
    assert errs.max() <= 1e-6, errs
