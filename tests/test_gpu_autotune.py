"""The stencil pass's per-level tiling and occupancy form
(amss_engine_set_level_tiling, amss_engine_set_level_occupancy) and their
autotuner (amss_b200.autotune): every tiling and form computes the same
numbers, bit for bit, and the tuner returns a valid choice for every level."""
import numpy as np
import pytest

import amss_b200
from amss_b200 import autotune
from amss_b200.hierarchy import box_in_box
import amr as OA

pytestmark = pytest.mark.gpu


def _hier():
    return box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)


def _run(H, init, dt0, tiling, precision="fp64"):
    e = amss_b200.Engine.from_hierarchy(H, precision=precision, eps=0.1)
    for i, st in enumerate(init):
        e.set_state(i, st)
    for lv, (w, z, o) in tiling.items():
        e.set_level_tiling(lv, w, z)
        e.set_level_occupancy(lv, o)
        assert e.level_tiling(lv)[:2] == (w, z) and e.level_occupancy(lv) == o
    e.run_coarse_graph(dt0, nsteps=1, replays=2)
    assert e.sync() == 0
    out = [e.get_state(i) for i in range(len(H.blocks))]
    e.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tilings_give_identical_results(precision):
    H = _hier()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-8)
    dt0 = 0.25 * H.h0
    base = _run(H, init, dt0, {}, precision)
    for tiling in ({0: (16, 3, 1), 1: (8, 2, 0), 2: (0, 4, 1)}, {0: (32, 1, 0), 1: (0, 2, 1), 2: (12, 2, 1)}):
        got = _run(H, init, dt0, tiling, precision)
        for a, b in zip(got, base):
            assert np.array_equal(a, b)


def test_bad_tiling_is_rejected():
    H = _hier()
    e = amss_b200.Engine.from_hierarchy(H, precision="fp64", eps=0.1)
    with pytest.raises(amss_b200.AmssError):
        e.set_level_tiling(0, 4, 1)
    with pytest.raises(amss_b200.AmssError):
        e.set_level_tiling(0, 0, 0)
    with pytest.raises(amss_b200.AmssError):
        e.set_level_tiling(7, 0, 1)
    with pytest.raises(amss_b200.AmssError):
        e.set_level_occupancy(0, 2)
    e.close()


def test_tuner_picks_a_candidate_for_every_level(tmp_path):
    H = _hier()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-8)
    cache = str(tmp_path / "tiling.json")
    got = autotune.tune(H, init, 0.25 * H.h0, cache=cache, reps=2)
    assert sorted(got) == [0, 1, 2]
    for lv, (w, z, o, ms) in got.items():
        assert (w, z, o) in autotune.candidates(H, lv) and ms > 0
    again = autotune.tune(H, init, 0.25 * H.h0, cache=cache)   # from the cache, nothing re-timed
    assert {k: tuple(v[:3]) for k, v in again.items()} == {k: tuple(v[:3]) for k, v in got.items()}
