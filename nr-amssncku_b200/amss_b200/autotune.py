"""Autotuner of the stencil pass's tiling, per level.

The stencil pass (k_deriv) runs one CTA per (field, x-y tile, z-slab) work
item.  How its items fill the GPU depends on each level's block shapes: the
tile width W (H = 256 / W rows) sets the halo overhead and the item count, the
z-split trades a 7-plane prologue per slab for more, shorter items that fill
the last wave of CTAs better, and the occupancy form (two resident CTAs per SM,
or four in FP64 / three in FP32 with fewer registers and some spills) trades
spills for warps.  The tuner times each
candidate on a scratch engine holding the same hierarchy and state (CUDA
events around graph replays of that level's RK4 step; the live engine is not
touched), keeps the fastest per level, and caches the choice in a JSON file
keyed by the level's block shapes, the precision and the formulation, so a
hierarchy of the same shapes is tuned once.  Results never depend on the
tiling: every candidate computes the same numbers.
"""
import json
import os

import numpy as np

from .engine import Engine

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "amss_b200", "tiling.json")


def level_key(H, level, precision, formulation):
    shapes = sorted(tuple(H.blocks[i].ex) for p in H.levels[level] for i in p.blocks)
    return f"{precision}/{formulation}/" + ";".join("x".join(map(str, s)) for s in shapes)


def candidates(H, level):
    """(tile width, z-split, occupancy) worth timing for a level: the default
    width and the widths that cut the level's smallest block width into 1-3
    near-equal tiles, each with 1-4 z-slabs, in both occupancy forms."""
    wmin = min(H.blocks[i].ex[0] for p in H.levels[level] for i in p.blocks)
    widths = {0}
    for parts in (1, 2, 3):
        w = -(-wmin // parts)
        if 8 <= w <= 64:
            widths.add(w)
    for w in (16, 32):
        if w <= wmin:
            widths.add(w)
    return [(w, z, o) for w in sorted(widths) for z in (1, 2, 3, 4) for o in (0, 1)]


def _time_level(eng, level, dt, reps):
    import torch
    stream = torch.cuda.ExternalStream(eng.stream)
    eng.run_graph(level, dt, nsteps=1, replays=1)   # warm-up (and graph instantiation)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    eng.run_graph(level, dt, nsteps=1, replays=reps)
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / reps


def tune(H, states, dt0, precision="fp64", formulation="bssn", eps=0.1, symmetry=0, cache=DEFAULT_CACHE,
         reps=3, levels=None):
    """{level: (tile_w, zsplit, occupancy, ms per step)} for the hierarchy,
    from the cache where an entry exists, else measured on a scratch engine
    (and stored)."""
    book = {}
    if cache and os.path.exists(cache):
        with open(cache) as f:
            book = json.load(f)
    out, todo = {}, []
    for lv in (range(len(H.levels)) if levels is None else levels):
        k = level_key(H, lv, precision, formulation)
        if k in book and len(book[k]) == 4:
            out[lv] = tuple(book[k])
        else:
            todo.append(lv)
    if todo:
        eng = Engine.from_hierarchy(H, precision=precision, eps=eps, symmetry=symmetry, formulation=formulation)
        try:
            for lv in todo:
                dt = dt0 / 2 ** lv
                best = None
                for w, z, o in candidates(H, lv):
                    for i, st in enumerate(states):
                        eng.set_state(i, st)
                    eng.set_level_tiling(lv, w, z)
                    eng.set_level_occupancy(lv, o)
                    ms = _time_level(eng, lv, dt, reps)
                    if best is None or ms < best[3]:
                        best = (w, z, o, ms)
                eng.set_level_tiling(lv, 0, 1)
                eng.set_level_occupancy(lv, 0)
                out[lv] = best
                book[level_key(H, lv, precision, formulation)] = list(best)
        finally:
            eng.close()
        if cache:
            os.makedirs(os.path.dirname(cache), exist_ok=True)
            with open(cache, "w") as f:
                json.dump(book, f, indent=1, sort_keys=True)
    return out


def apply(eng, choices):
    """Set the tuned tiling and occupancy on a live engine."""
    for lv, (w, z, o, _) in choices.items():
        eng.set_level_tiling(lv, w, z)
        eng.set_level_occupancy(lv, o)
