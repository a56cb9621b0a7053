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


# ---- constraint monitor (Parallel::L2Norm, Parallel.C:4214-4243) -----------

import oracle as O


def _oracle_level_norms(H, states, level, patch=None):
    """sqrt(sum c^2 dV) over the owned cells of the level's blocks inside their
    patch (buffer included), residuals from the oracle's compute_rhs_bssn co=0."""
    sums = np.zeros(7)
    for i, b in enumerate(H.blocks):
        if b.level != level or (patch is not None and b.patch != patch):
            continue
        X, Y, Z = H.coords(b)
        cons = O.compute_rhs_bssn(X, Y, Z, states[i], co=0, eps=0.1)[4]
        p = H.levels[level][b.patch]
        lo = [max(b.own_lo[d], p.ext_lo[d]) - b.org[d] for d in range(3)]
        hi = [min(b.own_hi[d], p.ext_hi[d]) - b.org[d] for d in range(3)]
        c = cons[:, lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        dv = (X[1] - X[0]) * (Y[1] - Y[0]) * (Z[1] - Z[0])
        sums += (c * c).sum(axis=(1, 2, 3)) * dv
    return np.sqrt(sums)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_constraint_norms_match_oracle(precision):
    H = small_hierarchy()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-6)
    e = amss_b200.Engine.from_hierarchy(H, precision=precision, eps=0.1)
    for i, st in enumerate(init):
        e.set_state(i, st)
    e.coarse_step(0.25 * H.h0)
    assert e.sync() == 0
    states = [e.get_state(i) for i in range(len(H.blocks))]
    for lv in range(len(H.levels)):
        got = e.constraint_norms(lv)
        ref = _oracle_level_norms(H, states, lv)
        assert np.all(ref > 0)
        np.testing.assert_allclose(got[:7], ref, rtol=1e-12, atol=0)
        assert got[7] == 0.0
    e.close()


def test_constraint_norms_first_patch():
    """Constraint_Out takes each level's first patch only (bssn_class.C:7475):
    on a level of two patches the first-patch norms are those of patch 0's
    blocks, the all-patch norms add patch 1's."""
    H = box_in_box(40, 10.0, [(4.5, 0.5, 0.0), (-4.5, -0.5, 0.0)], 2, box_cells=16, seed=2, block_min=10,
                   block_max=16)
    assert len(H.levels[1]) == 2
    init = OA.initial_state(H, [0.5, 0.5], [[4.5, 0.5, 0.0], [-4.5, -0.5, 0.0]], noise=1e-6)
    e = amss_b200.Engine.from_hierarchy(H, eps=0.1)
    try:
        for i, st in enumerate(init):
            e.set_state(i, st)
        states = [e.get_state(i) for i in range(len(H.blocks))]
        got = e.constraint_norms(1, first_patch=True)
        np.testing.assert_allclose(got[:7], _oracle_level_norms(H, states, 1, patch=0), rtol=1e-12, atol=0)
        allp = e.constraint_norms(1)
        np.testing.assert_allclose(allp[:7], _oracle_level_norms(H, states, 1), rtol=1e-12, atol=0)
        assert np.all(allp[:7] > got[:7])
        # one patch: the two agree
        np.testing.assert_array_equal(e.constraint_norms(0, first_patch=True), e.constraint_norms(0))
    finally:
        e.close()


def test_z4c_constraint_norms_match_oracle():
    """Z4c: the residuals of the first 24 fields (constraint_bssn) plus the
    L2 norm of Theta (Z4c_class.C:2491-2510)."""
    H = small_hierarchy()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-6, nf=25)
    e = amss_b200.Engine.from_hierarchy(H, precision="fp64", eps=0.1, formulation="z4c")
    for i, st in enumerate(init):
        e.set_state(i, st)
    e.coarse_step(0.25 * H.h0)
    assert e.sync() == 0
    states = [e.get_state(i) for i in range(len(H.blocks))]
    for lv in range(len(H.levels)):
        got = e.constraint_norms(lv)
        ref = _oracle_level_norms(H, [np.ascontiguousarray(s[:24]) for s in states], lv)
        np.testing.assert_allclose(got[:7], ref, rtol=1e-12, atol=0)
        th = 0.0
        for i, b in enumerate(H.blocks):
            if b.level != lv:
                continue
            p = H.levels[lv][b.patch]
            lo = [max(b.own_lo[d], p.ext_lo[d]) - b.org[d] for d in range(3)]
            hi = [min(b.own_hi[d], p.ext_hi[d]) - b.org[d] for d in range(3)]
            t = states[i][24, lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
            X, Y, Z = H.coords(b)
            th += float((t * t).sum()) * (X[1] - X[0]) * (Y[1] - Y[0]) * (Z[1] - Z[0])
        assert th > 0
        np.testing.assert_allclose(got[7], np.sqrt(th), rtol=1e-12, atol=0)
    e.close()


@pytest.mark.parametrize("symmetry", [0, 1])
def test_constraint_norms_bbox_blocks(symmetry):
    """Two blocks added by bbox inside one patch box, overlapping by 3 ghost
    cells: l2normhelper's bbox test (fmisc.f90:1286-1303) drops the ghosts of
    the shared side only.  Symmetry 1: the blocks start at the z = 0 plane
    (mirrored stencils, the plane's cells counted)."""
    n, h, lo = 24, 0.25, -3.0
    hi = lo + n * h
    mid = lo + 12 * h
    zlo = 0.0 if symmetry else lo
    zhi = zlo + n * h
    pbox = (lo, lo, zlo, hi, hi, zhi)
    boxes = [(lo, lo, zlo, mid + 3 * h, hi, zhi), (mid - 3 * h, lo, zlo, hi, hi, zhi)]
    e = amss_b200.Engine(precision="fp64", eps=0.1, symmetry=symmetry)
    sums = np.zeros(7)
    rng = np.random.default_rng(7)
    for bb in boxes:
        e.add_block(0, (15, n, n), bb, pbox)
    e.commit()
    Y = lo + (np.arange(n) + 0.5) * h
    Z = zlo + (np.arange(n) + 0.5) * h
    for bid, bb in enumerate(boxes):
        X = bb[0] + (np.arange(15) + 0.5) * h
        st = amss_b200.dropin.get_lousto_nbhs(X, Y, Z, [1.0], [[0.3, -0.2, 0.1]])
        st += 1e-6 * rng.uniform(-1, 1, st.shape)
        e.set_state(bid, st)
        cons = O.compute_rhs_bssn(X, Y, Z, st, symmetry=symmetry, co=0, eps=0.1)[4]
        i0, i1 = (0, 12) if bid == 0 else (3, 15)
        c = cons[:, :, :, i0:i1]
        sums += (c * c).sum(axis=(1, 2, 3)) * h ** 3
    got = e.constraint_norms(0)
    e.close()
    np.testing.assert_allclose(got[:7], np.sqrt(sums), rtol=1e-12, atol=0)


def test_hamiltonian_norm_converges_at_fourth_order():
    """Brill-Lindquist data (the exact solution, H = 0) on [2, 6]^3 away from
    the puncture at two resolutions: the monitor's Hamiltonian norm falls by
    2^4 per doubling.  Each block sits inside a larger patch box, so its 3
    ghost cells are left out and both norms cover exactly [2, 6]^3."""
    norms = []
    for cells in (16, 32):
        h = 4.0 / cells
        ex = cells + 6
        bb = (2.0 - 3 * h,) * 3 + (6.0 + 3 * h,) * 3
        e = amss_b200.Engine(precision="fp64", eps=0.1)
        e.add_block(0, (ex, ex, ex), bb, (-10.0,) * 3 + (10.0,) * 3)
        e.commit()
        X = bb[0] + (np.arange(ex) + 0.5) * h
        e.set_state(0, amss_b200.dropin.get_lousto_nbhs(X, X, X, [1.0], [[0.0, 0.0, 0.0]]))
        norms.append(e.constraint_norms(0)[0])
        e.close()
    order = np.log2(norms[0] / norms[1])
    assert 3.7 < order < 4.3, (norms, order)


# ---- point interpolation (Parallel::PatList_Interp_Points) -------------------

import interp as OI

BETA = [18, 19, 20]
BETA_SOA = [(-1, 1, 1), (1, -1, 1), (1, 1, -1)]


def test_interp_points_match_oracle():
    """Every level of the 3-level hierarchy after a coarse step: the shift
    (with its parities) and chi at seeded points, bit-identical to the
    oracle; points outside every patch of a level are not found there."""
    H = small_hierarchy()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-6)
    e = amss_b200.Engine.from_hierarchy(H, precision="fp64", eps=0.1)
    for i, st in enumerate(init):
        e.set_state(i, st)
    e.coarse_step(0.25 * H.h0)
    assert e.sync() == 0
    states = [e.get_state(i) for i in range(len(H.blocks))]
    rng = np.random.default_rng(11)
    fields = BETA + [0]
    soa = BETA_SOA + [(1, 1, 1)]
    for lv in range(len(H.levels)):
        pb = [H.phys_bbox(p) for p in H.levels[lv]]
        lo = np.min([b[:3] for b in pb], axis=0)
        hi = np.max([b[3:] for b in pb], axis=0)
        pts = rng.uniform(lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo), size=(40, 3))
        pts[0] = (1.2, 0.3, -0.4)
        got, found = e.interp_points(lv, pts, fields, soa)
        ref, rfound = OI.interp_points(OI.hierarchy_patches(H, lv, states), [tuple(p) for p in pts], fields, soa)
        assert list(found) == list(rfound)
        assert found.any() and not found.all()
        assert np.array_equal(got, np.array(ref))
    e.close()


def test_interp_points_symmetry_plane():
    """Symmetry 1, blocks added by bbox from the z = 0 plane: points within
    two cells of the plane interpolate through mirrored cells (betaz odd)."""
    n, h, lo = 24, 0.25, -3.0
    hi = lo + n * h
    mid = lo + 12 * h
    pbox = (lo, lo, 0.0, hi, hi, n * h)
    boxes = [(lo, lo, 0.0, mid + 3 * h, hi, n * h), (mid - 3 * h, lo, 0.0, hi, hi, n * h)]
    e = amss_b200.Engine(precision="fp64", eps=0.1, symmetry=1)
    for bb in boxes:
        e.add_block(0, (15, n, n), bb, pbox)
    e.commit()
    rng = np.random.default_rng(2)
    Y = lo + (np.arange(n) + 0.5) * h
    Z = (np.arange(n) + 0.5) * h
    blocks = []
    for bid, bb in enumerate(boxes):
        X = bb[0] + (np.arange(15) + 0.5) * h
        st = amss_b200.dropin.get_lousto_nbhs(X, Y, Z, [1.0], [[0.3, -0.2, 0.1]])
        st += 1e-3 * rng.uniform(-1, 1, st.shape)
        e.set_state(bid, st)
        blocks.append((bb, X, Y, Z, st))
    pts = np.column_stack([rng.uniform(lo, hi, 30), rng.uniform(lo, hi, 30), rng.uniform(0.0, 0.6, 30)])
    got, found = e.interp_points(0, pts, BETA, BETA_SOA)
    e.close()
    patches = [(pbox, [n, n, n], 0, blocks)]
    ref, rfound = OI.interp_points(patches, [tuple(p) for p in pts], BETA, BETA_SOA, symmetry=1)
    assert found.all() and all(rfound)
    assert np.array_equal(got, np.array(ref))


# ---- puncture tracking (bssn_class::Step, MAPBH 0) ---------------------------

@pytest.mark.parametrize("graph", [False, True])
def test_puncture_tracking_matches_oracle(graph):
    """A shift offset moves the puncture; after 2 coarse steps (8 steps of the
    finest level) the engine's tracked position equals the oracle's, bit for
    bit, eager or replayed from a CUDA graph."""
    H = small_hierarchy()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-6)
    for st in init:
        st[18] += 0.05
        st[19] -= 0.03
        st[20] += 0.02
    dt0 = 0.25 * H.h0
    start = [[1.2, 0.3, -0.4]]
    oh = OA.OracleHierarchy(H, eps=0.1)
    for i, st in enumerate(init):
        oh.set_state(i, st)
    oh.set_punctures(start)
    for _ in range(2):
        assert oh.coarse_step(dt0) == 0
    e = amss_b200.Engine.from_hierarchy(H, precision="fp64", eps=0.1)
    for i, st in enumerate(init):
        e.set_state(i, st)
    e.set_punctures(start)
    if graph:
        e.run_coarse_graph(dt0, nsteps=1, replays=2)
    else:
        for _ in range(2):
            e.coarse_step(dt0)
    assert e.sync() == 0
    got = e.punctures()
    e.close()
    ref = np.array(oh.porg0)
    assert np.array_equal(got, ref), (got, ref)
    assert abs(got[0, 0] - 1.2) > 5e-3   # it moved, against the shift


def test_puncture_tracking_mixed():
    """The mixed form tracks from its FP32 stages: within 1e-9 of the FP64
    oracle after 2 coarse steps (the puncture moves by about 1e-2)."""
    H = small_hierarchy()
    init = OA.initial_state(H, [1.0], [[1.2, 0.3, -0.4]], noise=1e-6)
    for st in init:
        st[18] += 0.05
        st[19] -= 0.03
        st[20] += 0.02
    dt0 = 0.25 * H.h0
    oh = OA.OracleHierarchy(H, eps=0.1)
    for i, st in enumerate(init):
        oh.set_state(i, st)
    oh.set_punctures([[1.2, 0.3, -0.4]])
    for _ in range(2):
        assert oh.coarse_step(dt0) == 0
    e = amss_b200.Engine.from_hierarchy(H, precision="mixed", eps=0.1)
    for i, st in enumerate(init):
        e.set_state(i, st)
    e.set_punctures([[1.2, 0.3, -0.4]])
    e.run_coarse_graph(dt0, nsteps=1, replays=2)
    assert e.sync() == 0
    got = e.punctures()
    e.close()
    assert np.abs(got - np.array(oh.porg0)).max() <= 1e-9


def test_final_substep_regions_in_use():
    """The coarse-step parity above runs with final-substep regions on both
    refined levels (the owned cells within 2 of the physical box)."""
    H = small_hierarchy()
    e = amss_b200.Engine.from_hierarchy(H, eps=0.1)
    try:
        # level 0: no regions; its ghosts are synchronised, so its owned cells
        own0 = sum(int(np.prod([H.blocks[bi].own_hi[d] - H.blocks[bi].own_lo[d] for d in range(3)]))
                   for p in H.levels[0] for bi in p.blocks)
        assert e.final_region(0) == (-1, own0)
        for lv in (1, 2):
            pad, pts = e.final_region(lv)
            assert pad == 2 and 0 < pts < H.points(lv)
    finally:
        e.close()


def test_single_level_step_updates_every_cell(fp64_reference):
    """amss_engine_step_level is not followed by RestrictProlong: its final
    substep still updates the buffer cells, as the oracle's level step does."""
    H, init, dt0, _ = fp64_reference
    oh = OA.OracleHierarchy(H, eps=0.1)
    e = amss_b200.Engine.from_hierarchy(H, eps=0.1)
    try:
        for i, st in enumerate(init):
            oh.set_state(i, st)
            e.set_state(i, st)
        dt = dt0 / 2
        assert oh.level_step(1, dt) == 0
        e.step(1, dt)
        assert e.sync() == 0
        ids = [i for p in H.levels[1] for i in p.blocks]
        errs = _errs([e.get_state(i) for i in ids], [oh.state(i) for i in ids])
        assert errs.max() <= 1e-12, errs
    finally:
        e.close()


def test_level_without_regions_matches_oracle():
    """Level 2's buffered box reaches level 1's physical boundary: level 1
    takes no regions in its final substep, level 2 does; two
    coarse steps against the oracle."""
    from amss_b200.hierarchy import Hierarchy
    H = Hierarchy(-8.0, 0.5)
    H.add_patch(0, (0, 0, 0), (32, 32, 32), 0, [[], [], []])
    H.add_patch(1, (24, 24, 24), (40, 40, 40), 6, [[32], [], []])
    H.add_patch(2, (54, 54, 54), (70, 70, 70), 6, [[], [62], []])
    init = OA.initial_state(H, [0.5], [[0.1, 0.05, 0.02]], noise=1e-8)
    dt0 = 0.25 * H.h0
    ref = _run_oracle(H, init, dt0, 2)
    e = amss_b200.Engine.from_hierarchy(H, eps=0.1)
    try:
        assert e.final_region(1)[0] == -1 and e.final_region(2)[0] == 2
    finally:
        e.close()
    got = _run_engine(H, init, dt0, 2)
    errs = _errs(got, ref)
    assert errs.max() <= 1e-12, errs
