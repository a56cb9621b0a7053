"""The final-substep regions of a coarse step (amss_engine_level_final_region),
planned without a device.

In a coarse step the final RK4 substep of a refined level updates only each
owned block's cells within 2 of its patch's physical box: RestrictProlong
(bssn_class.C:5724-5903) overwrites the other buffer cells before anything
reads them.  Commit grants this per level after checking every read of the
level's new state (the restriction out of it, restrict3: fine 2k-2 .. 2k+3;
the finer level's prolongation, prolong3: coarse k-3 .. k+3) and that the
prolongation into the level covers its buffer cells.  Checked here: the amr
bench hierarchy gets regions on every refined level with the expected cell
counts; the counts divide among ranks; a level whose child's buffer reaches
its physical boundary keeps no regions (its owned cells, whose ghosts the
sync fills)."""
import numpy as np

from amss_b200 import dist as D
from amss_b200.hierarchy import Hierarchy, box_in_box


def expected_points(H, lv, pad, blocks=None):
    n = 0
    for p in H.levels[lv]:
        for bi in p.blocks:
            if blocks is not None and bi not in blocks:
                continue
            b = H.blocks[bi]
            lo = [max(b.own_lo[d], p.lo[d] - pad, b.org[d]) for d in range(3)]
            hi = [min(b.own_hi[d], p.hi[d] + pad, b.org[d] + b.ex[d]) for d in range(3)]
            n += int(np.prod([max(0, hi[d] - lo[d]) for d in range(3)]))
    return n


def owned_points(H, lv):
    return sum(int(np.prod([H.blocks[bi].own_hi[d] - H.blocks[bi].own_lo[d] for d in range(3)]))
               for p in H.levels[lv] for bi in p.blocks)


def amr_hierarchy():
    return box_in_box(96, 48.0, [(-3.0, 0.0, 0.0), (3.0, 0.0, 0.0)], 7, box_cells=48, seed=1,
                      block_min=18, block_max=74)


def touching_hierarchy():
    """Level 2's buffered box reaches level 1's physical boundary (coarse
    cell 24), so level 2's prolongation reads level-1 cells 3 past it."""
    H = Hierarchy(-8.0, 0.5)
    H.add_patch(0, (0, 0, 0), (32, 32, 32), 0, [[], [], []])
    H.add_patch(1, (24, 24, 24), (40, 40, 40), 6, [[32], [], []])
    H.add_patch(2, (54, 54, 54), (70, 70, 70), 6, [[], [62], []])
    return H


def test_amr_levels_take_final_regions():
    H = amr_hierarchy()
    P = D.Plan.of(H, 0, 1, [0] * len(H.blocks))
    try:
        # level 0 has no regions; its ghost cells are synchronised, so the final
        # substep updates the owned cells
        assert owned_points(H, 0) < H.points(0)
        assert P.final_region(0) == (-1, owned_points(H, 0))
        for lv in range(1, len(H.levels)):
            pad, pts = P.final_region(lv)
            assert pad == 2
            assert pts == expected_points(H, lv, 2) < H.points(lv)
    finally:
        P.close()


def test_rank_plans_count_their_own_blocks():
    H = amr_hierarchy()
    owners = D.partition(H, 3)
    tot = {lv: 0 for lv in range(len(H.levels))}
    for r in range(3):
        P = D.Plan.of(H, r, 3, owners)
        try:
            for lv in range(1, len(H.levels)):
                pad, pts = P.final_region(lv)
                mine = {bi for bi, o in enumerate(owners) if o == r}
                assert pad == 2 and pts == expected_points(H, lv, 2, mine)
                tot[lv] += pts
        finally:
            P.close()
    assert all(tot[lv] == expected_points(H, lv, 2) for lv in range(1, len(H.levels)))


def test_level_read_past_its_pad_keeps_no_regions():
    H = touching_hierarchy()
    P = D.Plan.of(H, 0, 1, [0] * len(H.blocks))
    try:
        assert P.final_region(1) == (-1, owned_points(H, 1))
        assert P.final_region(2) == (2, expected_points(H, 2, 2))
    finally:
        P.close()


def test_blocks_added_by_bbox_keep_whole_arrays():
    """Blocks added by bounding box (each its own patch, cells numbered from
    0) have no same-level sync to rely on: their substeps cover whole arrays."""
    P = D.Plan(eps=0.1)
    try:
        a = [-2.0, -2.0, -2.0, 1.0, 1.0, 1.0]
        b = [0.0, -2.0, -2.0, 3.0, 1.0, 1.0]
        P.add_block(0, (12, 12, 12), a, a)
        P.add_block(0, (12, 12, 12), b, b)
        P.commit()
        assert P.final_region(0) == (-1, 2 * 12 ** 3)
    finally:
        P.close()
