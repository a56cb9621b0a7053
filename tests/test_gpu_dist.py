"""The hierarchy divided among ranks gives the one-engine result bit for bit.

Ranks run as engines of one process (amss_b200.dist.LocalGroup), one host
thread each, all on the one GPU of this test: every rank allocates and steps
only its own blocks, and every ghost, restriction and prolongation segment
between blocks of different ranks goes through the staging regions and the
device-to-device exchange.  No kernel waits on another rank's kernel (stream
order, events and a host barrier order the exchange), so ranks sharing a GPU
is safe.  Two coarse steps of the three-level test hierarchy (uneven blocks,
buffer zones, time interpolation) must equal a single engine's exactly, in
FP64 and in the mixed form; the ranks' constraint sums add up to the single
engine's norms."""
import numpy as np
import pytest

import amss_b200
from amss_b200 import dist as D
from amss_b200.hierarchy import box_in_box
import amr as OA

pytestmark = pytest.mark.gpu


def small_hierarchy():
    return box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)


def _single(H, init, dt0, steps, **kw):
    e = amss_b200.Engine.from_hierarchy(H, eps=0.1, **kw)
    for i, st in enumerate(init):
        e.set_state(i, st)
    for _ in range(steps):
        e.coarse_step(dt0)
    assert e.sync() == 0
    out = [e.get_state(i) for i in range(len(H.blocks))]
    norms = [e.constraint_norms(lv) for lv in range(len(H.levels))]
    e.close()
    return out, norms


def _group(H, init, dt0, steps, owners, nranks, **kw):
    G = D.LocalGroup(H, owners, nranks, timeout=30.0, eps=0.1, **kw)
    try:
        for i, st in enumerate(init):
            G.set_state(i, st)
        G.coarse_step(dt0, steps=steps)
        assert G.sync() == 0
        out = [G.get_state(i) for i in range(len(H.blocks))]
        norms = [G.constraint_norms(lv) for lv in range(len(H.levels))]
        cross = sum(x["ncross"] for x in D.xfer_tables(G.engines[0]))
    finally:
        G.close()
    return out, norms, cross


@pytest.fixture(scope="module")
def case():
    H = small_hierarchy()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-8)
    return H, init, 0.25 * H.h0


@pytest.mark.parametrize("precision,nranks,mode", [("fp64", 2, "balanced"), ("fp64", 3, "round_robin"),
                                                   ("mixed", 2, "balanced")])
def test_ranks_equal_one_engine(case, precision, nranks, mode):
    H, init, dt0 = case
    ref, rnorm = _single(H, init, dt0, 2, precision=precision)
    owners = D.partition(H, nranks, mode)
    got, gnorm, cross = _group(H, init, dt0, 2, owners, nranks, precision=precision)
    assert cross > 0
    bad = [i for i, (g, r) in enumerate(zip(got, ref)) if not np.array_equal(g, r)]
    assert bad == [], bad
    for a, b in zip(gnorm, rnorm):
        assert np.allclose(a, b, rtol=1e-12, atol=0)


def test_z4c_ranks_equal_one_engine(case):
    """25 fields (Theta last): the staging regions follow the field count."""
    H, init, dt0 = case
    init25 = [np.concatenate([s, 1e-8 * np.ones((1,) + s.shape[1:])]) for s in init]
    ref, _ = _single(H, init25, dt0, 1, formulation="z4c")
    got, _, cross = _group(H, init25, dt0, 1, D.partition(H, 2), 2, formulation="z4c")
    assert cross > 0 and all(np.array_equal(g, r) for g, r in zip(got, ref))


def test_rank_without_blocks_on_a_level(case):
    """Rank 1 holds no block of the finest level: it still takes part in
    that level's exchanges (restriction into its level-1 blocks)."""
    H, init, dt0 = case
    ref, _ = _single(H, init, dt0, 1)
    owners = D.partition(H, 2)
    for p in H.levels[2]:
        for bi in p.blocks:
            owners[bi] = 0
    got, _, _ = _group(H, init, dt0, 1, owners, 2)
    assert all(np.array_equal(g, r) for g, r in zip(got, ref))


def test_rank_engine_refuses_whole_hierarchy_calls(case):
    H, init, dt0 = case
    owners = D.partition(H, 2)
    e = amss_b200.Engine.from_hierarchy(H, rank=0, nranks=2, owners=owners, eps=0.1)
    try:
        other = owners.index(1)
        with pytest.raises(amss_b200.AmssError):
            e.get_state(other)
        with pytest.raises(amss_b200.AmssError):
            e.run_coarse_graph(dt0, 1)
        with pytest.raises(amss_b200.AmssError):
            e.set_punctures([[1.2, 0.3, -0.4]])
        # no transport: the first exchange is refused, not skipped
        with pytest.raises(amss_b200.AmssError):
            e.coarse_step(dt0)
    finally:
        e.close()
