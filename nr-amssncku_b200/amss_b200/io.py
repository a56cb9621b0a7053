"""The reference's on-disk formats for the evolution state.

* Binary dumps (Parallel::Dump_Data, Parallel.C:1221-1373, written by
  Parallel::writefile, :1049-1071): one file per patch and field,
  `{out}/[tag_]Lev{lev:02d}-{patch:02d}_{name}_{count:05d}.bin` with count =
  int(time / dt + 0.5), holding time (double), nx, ny, nz (int32), xmin, xmax,
  ymin, ymax, zmin, zmax (double) and the patch's nx*ny*nz doubles, x fastest.
  A patch is its extended box (buffer cells included on refined levels), its
  data the owned cells of its blocks (ghost cells dropped).  The reference's
  plot_binary_data.py reads these files.
* Checkpoints (checkpoint::writecheck_cgh / readcheck_cgh, checkpoint.C:132-300):
  `{prefix}_cgh.CHK` holding time, levels, movls, BH_num (int32), grids[levels]
  (int32), Lt[levels] (double), then per level per grid bbox[6] (double),
  shape[3] (int32), handle[3] (double) and per puncture Porgls[3] (double),
  then per level, per patch, per variable of the CheckList -- StateList then
  OldStateList (bssn_class.C:682-683), i.e. the current and the previous time
  level of the 24 fields -- the patch's data as in a dump.

Fields are stored as the engine holds them, which is the reference's storage:
chi - 1 as phi, the diagonal metric less 1, Lap - 1.
"""
import os
import struct

import numpy as np

from .hierarchy import from_boxes

# StateList (bssn_class.C:437-460) and OldStateList (:412-435) variable names
BASE_NAMES = ["phi", "trK", "gxx", "gxy", "gxz", "gyy", "gyz", "gzz", "Axx", "Axy", "Axz", "Ayy", "Ayz", "Azz",
              "Gmx", "Gmy", "Gmz", "Lap", "Sfx", "Sfy", "Sfz", "dtSfx", "dtSfy", "dtSfz"]
STATE_VARS = [n + "0" for n in BASE_NAMES]
OLD_VARS = [n + "o" for n in BASE_NAMES]


def _view(org, arr, lo, hi):
    return arr[(slice(None),) + tuple(slice(lo[d] - org[d], hi[d] - org[d]) for d in (2, 1, 0))]


def patch_array(H, level, pid, block_data):
    """The patch's extended box assembled from its blocks' owned cells:
    (nf, nz, ny, nx).  block_data(i) gives block i's array (nf, ez, ey, ex)."""
    p = H.levels[level][pid]
    lo, hi = p.ext_lo, p.ext_hi
    out = None
    for bi in p.blocks:
        b = H.blocks[bi]
        a = block_data(bi)
        if out is None:
            out = np.empty((a.shape[0],) + tuple(hi[d] - lo[d] for d in (2, 1, 0)))
        _view(lo, out, b.own_lo, b.own_hi)[...] = _view(b.org, a, b.own_lo, b.own_hi)
    return out


def scatter_patch(H, level, pid, data, set_block):
    """The inverse of patch_array: every block's array (ghost cells included,
    they lie inside the patch) cut from the patch data and handed to
    set_block(i, array)."""
    p = H.levels[level][pid]
    for bi in p.blocks:
        b = H.blocks[bi]
        hi = tuple(b.org[d] + b.ex[d] for d in range(3))
        set_block(bi, np.ascontiguousarray(_view(p.ext_lo, data, b.org, hi)))


def _bbox(H, level, lo, hi):
    h = H.h(level)
    return [H.x0 + lo[d] * h for d in range(3)] + [H.x0 + hi[d] * h for d in range(3)]


def write_dump(out_dir, H, level, time, dt, block_data, fields=None, tag=None):
    """Parallel::Dump_Data of one level: returns the files written."""
    os.makedirs(out_dir, exist_ok=True)
    count = int(time / dt + 0.5)
    files = []
    for pid, p in enumerate(H.levels[level]):
        data = patch_array(H, level, pid, block_data)
        bb = _bbox(H, level, p.ext_lo, p.ext_hi)
        nz, ny, nx = data.shape[1:]
        for f in (range(data.shape[0]) if fields is None else fields):
            name = (STATE_VARS + ["TZ0"])[f]
            fn = f"{tag}_" if tag else ""
            fn += f"Lev{level:02d}-{pid:02d}_{name}_{count:05d}.bin"
            path = os.path.join(out_dir, fn)
            with open(path, "wb") as fh:
                fh.write(struct.pack("<d3i6d", time, nx, ny, nz, bb[0], bb[3], bb[1], bb[4], bb[2], bb[5]))
                fh.write(np.ascontiguousarray(data[f], dtype="<f8").tobytes())
            files.append(path)
    return files


def read_dump(path):
    """A dump file as the reference's plot_binary_data.py reads it."""
    with open(path, "rb") as fh:
        time = np.fromfile(fh, dtype=np.float64, count=1)[0]
        nx, ny, nz = np.fromfile(fh, dtype=np.int32, count=3)
        box = np.fromfile(fh, dtype=np.float64, count=6)
        data = np.fromfile(fh, dtype=np.float64)
    return dict(time=float(time), shape=(int(nx), int(ny), int(nz)), bbox=box.tolist(),
                data=data.reshape(int(nz), int(ny), int(nx)))


def write_checkpoint(prefix, H, time, level_times, regridder, time_level, movls=1):
    """checkpoint::writecheck_cgh: `time_level(block, back)` gives a block's
    state back = 0 (StateList) or 1 (OldStateList) steps ago; regridder holds
    the boxes, centres and Porgls of the levels >= 1 (level 0 is one box)."""
    nlev = len(H.levels)
    nbh = len(regridder.porgls[0]) if regridder.porgls else 0
    grids = [1] + [len(b) for b in regridder.boxes]
    path = f"{prefix}_cgh.CHK"
    with open(path, "wb") as fh:
        fh.write(struct.pack("<d3i", time, nlev, movls, nbh))
        fh.write(struct.pack(f"<{nlev}i", *grids))
        fh.write(struct.pack(f"<{nlev}d", *level_times))
        for lev in range(nlev):
            if lev == 0:
                p = H.levels[0][0]
                boxes = [[list(p.lo), list(p.hi)]]
                handles = [[H.x0 + 0.5 * (p.lo[d] + p.hi[d]) * H.h0 for d in range(3)]]
                porgls = regridder.porgls[0] if regridder.porgls else []
            else:
                boxes, handles, porgls = regridder.boxes[lev - 1], regridder.handles[lev - 1], regridder.porgls[lev - 1]
            for (lo, hi), hd in zip(boxes, handles):
                fh.write(struct.pack("<6d", *_bbox(H, lev, lo, hi)))
                fh.write(struct.pack("<3i", *[hi[d] - lo[d] for d in range(3)]))
                fh.write(struct.pack("<3d", *hd))
            for pb in porgls:
                fh.write(struct.pack("<3d", *pb))
        for lev in range(nlev):
            for pid in range(len(H.levels[lev])):
                for back in (0, 1):
                    data = patch_array(H, lev, pid, lambda bi: time_level(bi, back))
                    for f in range(data.shape[0]):
                        fh.write(np.ascontiguousarray(data[f], dtype="<f8").tobytes())
    return path


def read_checkpoint(prefix, nf=24):
    """checkpoint::readcheck_cgh: the header and, per level and patch, the
    current and previous data.  The hierarchy is rebuilt from the boxes with the
    block split of amss_b200.hierarchy (seed 1, blocks of 24..80 cells unless the
    caller rebuilds it otherwise)."""
    path = f"{prefix}_cgh.CHK"
    with open(path, "rb") as fh:
        raw = fh.read()
    off = 0

    def take(fmt):
        nonlocal off
        vals = struct.unpack_from(fmt, raw, off)
        off += struct.calcsize(fmt)
        return vals

    time, nlev, movls, nbh = take("<d3i")
    grids = list(take(f"<{nlev}i"))
    lt = list(take(f"<{nlev}d"))
    bboxes, shapes, handles, porgls = [], [], [], []
    for lev in range(nlev):
        bb, sh, hd = [], [], []
        for _ in range(grids[lev]):
            bb.append(list(take("<6d")))
            sh.append(list(take("<3i")))
            hd.append(list(take("<3d")))
        bboxes.append(bb)
        shapes.append(sh)
        handles.append(hd)
        porgls.append([list(take("<3d")) for _ in range(nbh)])
    return dict(time=time, levels=nlev, movls=movls, nbh=nbh, grids=grids, lt=lt, bbox=bboxes, shape=shapes,
                handle=handles, porgls=porgls, raw=raw, data_offset=off, nf=nf)


def hierarchy_from_checkpoint(ck, seed=1, block_min=24, block_max=80):
    """The hierarchy of a checkpoint's boxes, and a Regridder-compatible state
    (boxes, handles, porgls of the levels >= 1)."""
    bb0, sh0 = ck["bbox"][0][0], ck["shape"][0][0]
    h0 = (bb0[3] - bb0[0]) / sh0[0]
    x0 = bb0[0]
    levels = []
    for lev in range(1, ck["levels"]):
        h = h0 / 2 ** lev
        boxes = []
        for bb, sh in zip(ck["bbox"][lev], ck["shape"][lev]):
            lo = [int(round((bb[d] - x0) / h)) for d in range(3)]
            boxes.append([lo, [lo[d] + sh[d] for d in range(3)]])
        levels.append(boxes)
    H = from_boxes(x0, h0, tuple(sh0), levels, seed, block_min, block_max)
    return H


def checkpoint_patches(ck, H):
    """Yield (level, patch, back, data[nf, nz, ny, nx]) in file order."""
    off = ck["data_offset"]
    nf = ck["nf"]
    for lev in range(ck["levels"]):
        for pid, p in enumerate(H.levels[lev]):
            shp = tuple(p.ext_hi[d] - p.ext_lo[d] for d in (2, 1, 0))
            n = int(np.prod(shp))
            for back in (0, 1):
                data = np.frombuffer(ck["raw"], dtype="<f8", count=nf * n, offset=off).reshape((nf,) + shp)
                off += 8 * nf * n
                yield lev, pid, back, data


def save_engine(prefix, eng, H, regridder, time, dt0, movls=1):
    """checkpoint::writecheck_cgh of an engine: the current and previous time
    level of every block, each level's time (its steps x its step size)."""
    eng.sync()
    lt = [eng.level_steps(lv) * dt0 / 2 ** lv for lv in range(len(H.levels))]
    return write_checkpoint(prefix, H, time, lt, regridder, lambda bi, back: eng.get_time_level(bi, back), movls)


def load_engine(prefix, dt0, seed=1, block_min=24, block_max=80, **engine_kw):
    """An engine resumed from a checkpoint: (engine, hierarchy, time, the
    moving-box state as a Regridder)."""
    from .engine import Engine
    from .regrid import Regridder
    ck = read_checkpoint(prefix, nf=25 if engine_kw.get("formulation") == "z4c" else 24)
    H = hierarchy_from_checkpoint(ck, seed, block_min, block_max)
    eng = Engine.from_hierarchy(H, **engine_kw)
    for lev, pid, back, data in checkpoint_patches(ck, H):
        scatter_patch(H, lev, pid, data, lambda bi, a: eng.set_time_level(bi, back, a))
    for lv in range(ck["levels"]):
        eng.set_level_steps(lv, int(round(ck["lt"][lv] / (dt0 / 2 ** lv))))
    r = Regridder(H, ck["porgls"][0] if ck["nbh"] else [], movls=ck["movls"])
    r.handles = [list(map(list, ck["handle"][lv])) for lv in range(1, ck["levels"])]
    r.porgls = [list(map(list, ck["porgls"][lv])) for lv in range(1, ck["levels"])]
    return eng, H, ck["time"], r
