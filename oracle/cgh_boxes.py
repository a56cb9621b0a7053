"""CPU restatement of the reference's box merging of a refined level (test
infrastructure only).

cgh::compose_cgh (cgh.C:1211-1230) merges the grid boxes of a level only when
the level has fewer than 3 of them: Parallel::merge_gsl (Parallel.C:4941-4995)
walks the list, D from the head and B after it, and at the first pair that
merge_gs (:4997-5086, Cell) accepts removes both and appends their bounding
box to the end of the list, then starts over.  merge_gs accepts two boxes that
touch or overlap on every axis (uub - llb >= 0) when the merged box is filled
well enough: (vd + vb - vo) / vt > ratio, ratio = 0.75 (cgh.h:41).  Pairs that
still overlap afterwards are cut apart by Parallel::cut_gsl and touching ones
get ghost regions from add_ghost_touch; this restatement reports those cases
instead of reproducing them.

Boxes are [lo, hi) in the level's global cell indices; the reference's double
bboxes are these times the cell size, so the volume ratio is the same.
"""
RATIO = 0.75


def _merge_gs(d, b):
    lo = [max(d[0][i], b[0][i]) for i in range(3)]
    hi = [min(d[1][i], b[1][i]) for i in range(3)]
    if any(hi[i] - lo[i] < 0 for i in range(3)):
        return None
    vd = vb = vt = vo = 1.0
    for i in range(3):
        vt *= max(d[1][i], b[1][i]) - min(d[0][i], b[0][i])
        vo *= hi[i] - lo[i]
        vd *= d[1][i] - d[0][i]
        vb *= b[1][i] - b[0][i]
    if (vd + vb - vo) / vt > RATIO:
        return [[min(d[0][i], b[0][i]) for i in range(3)], [max(d[1][i], b[1][i]) for i in range(3)]]
    return None


def merge_gsl(boxes):
    """Parallel::merge_gsl on a list of [lo, hi) boxes."""
    boxes = [[list(lo), list(hi)] for lo, hi in boxes]
    while True:
        hit = None
        for a in range(len(boxes)):
            for c in range(a + 1, len(boxes)):
                m = _merge_gs(boxes[a], boxes[c])
                if m is not None:
                    hit = (a, c, m)
                    break
            if hit:
                break
        if not hit:
            return boxes
        a, c, m = hit
        boxes = [bx for k, bx in enumerate(boxes) if k not in (a, c)] + [m]


def compose_level(boxes):
    """The patches cgh::compose_cgh makes of a level's grid boxes, and the
    pairs left overlapping or touching (which cut_gsl / add_ghost_touch would
    reshape; [] when there are none)."""
    out = merge_gsl(boxes) if len(boxes) < 3 else [[list(lo), list(hi)] for lo, hi in boxes]
    left = []
    for a in range(len(out)):
        for c in range(a + 1, len(out)):
            if all(min(out[a][1][i], out[c][1][i]) - max(out[a][0][i], out[c][0][i]) >= 0 for i in range(3)):
                left.append((a, c))
    return out, left
