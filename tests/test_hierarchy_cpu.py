"""The engine's patches against the reference's composition of a level's grid
boxes (cgh::compose_cgh with Parallel::merge_gsl, restated independently in
oracle/cgh_boxes.py), without a GPU.

On the benched workload (two punctures, seven levels) and on the reference's
own parameter file for it, every level gets exactly the reference's patches.
The two rules differ by design where the engine needs patches that do not
touch through their buffers: boxes a few cells apart (the reference keeps two
patches whose buffers overlap; the engine merges them), and three or more
boxes on a level (the reference merges none)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import cgh_boxes as CB   # noqa: E402
from amss_b200 import parfile   # noqa: E402
from amss_b200.hierarchy import merge_boxes   # noqa: E402


def _same(a, b):
    return sorted(map(str, a)) == sorted(map(str, b))


def test_benched_workload_patches_are_the_references():
    import bench
    H = bench.workload("amr")["H"]
    for boxes in H.grid_boxes:
        ref, left = CB.compose_level(boxes)
        assert left == []
        assert _same(merge_boxes(boxes), ref)
    # and the patches the hierarchy actually holds
    for lv, boxes in enumerate(H.grid_boxes, start=1):
        ref, _ = CB.compose_level(boxes)
        assert _same([[list(p.lo), list(p.hi)] for p in H.levels[lv]], ref)


def test_reference_parfile_patches_are_the_references():
    cfg = parfile.load(os.path.join(ROOT, "tests", "golden", "amr_workload.par"))
    H = cfg.hierarchy
    for lv, boxes in enumerate(H.grid_boxes, start=1):
        ref, left = CB.compose_level(boxes)
        assert left == [] and _same([[list(p.lo), list(p.hi)] for p in H.levels[lv]], ref)


@pytest.mark.parametrize("overlap,fill_ok", [(10, True), (0, True)])
def test_overlapping_and_touching_aligned_boxes_merge_in_both(overlap, fill_ok):
    a = [[0, 0, 0], [48, 48, 48]]
    b = [[48 - overlap, 0, 0], [96 - overlap, 48, 48]]
    ref, left = CB.compose_level([a, b])
    assert left == [] and len(ref) == 1
    assert _same(merge_boxes([a, b]), ref)


def test_documented_differences():
    # a gap of 6 cells: the reference keeps two patches, whose 6-cell buffers overlap
    a = [[0, 0, 0], [48, 48, 48]]
    b = [[54, 0, 0], [102, 48, 48]]
    ref, _ = CB.compose_level([a, b])
    assert len(ref) == 2 and len(merge_boxes([a, b])) == 1
    # three boxes in a row, overlapping: the reference merges none of them
    c = [[90, 0, 0], [138, 48, 48]]
    b2 = [[40, 0, 0], [88, 48, 48]]
    ref3, left3 = CB.compose_level([a, b2, c])
    assert len(ref3) == 3 and left3 and len(merge_boxes([a, b2, c])) == 1
