"""The reference's binary dump and checkpoint formats (amss_b200.io) on CPU:
byte layout read back by restatements of the reference's readers
(plot_binary_data.py for dumps, checkpoint::readcheck_cgh for checkpoints),
patch assembly from block owned cells, and a write -> read round trip."""
import struct

import numpy as np

from amss_b200 import io
from amss_b200.hierarchy import box_in_box
from amss_b200.regrid import Regridder


def _hier():
    return box_in_box(40, 10.0, [(1.2, 0.3, -0.4)], 3, box_cells=32, seed=4, block_min=14, block_max=28)


def _global_field(H, level, f, g):
    """A value per global cell of a level, identical in every copy of the cell."""
    return np.sin(0.37 * g[0] + 0.11 * f) + np.cos(0.23 * g[1]) * 0.5 + 0.01 * g[2] + level


def _block_arrays(H, nf=24, shift=0.0):
    out = []
    for b in H.blocks:
        k, j, i = np.meshgrid(*[np.arange(b.org[d], b.org[d] + b.ex[d]) for d in (2, 1, 0)], indexing="ij")
        out.append(np.stack([_global_field(H, b.level, f, (i, j, k)) + shift for f in range(nf)]))
    return out


def test_dump_layout_and_patch_assembly(tmp_path):
    H = _hier()
    arrs = _block_arrays(H)
    files = io.write_dump(str(tmp_path), H, 1, time=0.75, dt=0.125, block_data=lambda bi: arrs[bi], fields=[0, 17])
    p = H.levels[1][0]
    assert [f.split("/")[-1] for f in files] == ["Lev01-00_phi0_00006.bin", "Lev01-00_Lap0_00006.bin"]
    raw = open(files[1], "rb").read()
    t, nx, ny, nz = struct.unpack_from("<d3i", raw, 0)
    box = struct.unpack_from("<6d", raw, 20)
    assert t == 0.75 and (nx, ny, nz) == tuple(p.ext_hi[d] - p.ext_lo[d] for d in range(3))
    h = H.h(1)
    assert np.allclose(box, [H.x0 + p.ext_lo[0] * h, H.x0 + p.ext_hi[0] * h, H.x0 + p.ext_lo[1] * h,
                             H.x0 + p.ext_hi[1] * h, H.x0 + p.ext_lo[2] * h, H.x0 + p.ext_hi[2] * h])
    data = np.frombuffer(raw, dtype="<f8", offset=68).reshape(nz, ny, nx)
    k, j, i = np.meshgrid(*[np.arange(p.ext_lo[d], p.ext_hi[d]) for d in (2, 1, 0)], indexing="ij")
    assert np.array_equal(data, _global_field(H, 1, 17, (i, j, k)))
    r = io.read_dump(files[1])
    assert r["time"] == 0.75 and np.array_equal(r["data"], data)


def _read_cgh_header(raw):
    """checkpoint::readcheck_cgh's read sequence (checkpoint.C:196-260)."""
    off = 0
    time, levels, movls, bh = struct.unpack_from("<d3i", raw, off); off += 20
    grids = struct.unpack_from(f"<{levels}i", raw, off); off += 4 * levels
    lt = struct.unpack_from(f"<{levels}d", raw, off); off += 8 * levels
    boxes = []
    for lev in range(levels):
        for _ in range(grids[lev]):
            bb = struct.unpack_from("<6d", raw, off); off += 48
            sh = struct.unpack_from("<3i", raw, off); off += 12
            hd = struct.unpack_from("<3d", raw, off); off += 24
            boxes.append((lev, bb, sh, hd))
        off += 24 * bh
    return time, levels, movls, grids, lt, boxes, off


def test_checkpoint_layout_and_round_trip(tmp_path):
    H = _hier()
    cur, old = _block_arrays(H), _block_arrays(H, shift=1.0)
    r = Regridder(H, [(1.2, 0.3, -0.4)])
    prefix = str(tmp_path / "bssn")
    path = io.write_checkpoint(prefix, H, 0.5, [0.5, 0.5, 0.5], r, lambda bi, back: (cur, old)[back][bi])
    raw = open(path, "rb").read()
    time, levels, movls, grids, lt, boxes, off = _read_cgh_header(raw)
    assert (time, levels, movls, grids, lt) == (0.5, 3, 1, (1, 1, 1), (0.5, 0.5, 0.5))
    npatch = sum(int(np.prod([p.ext_hi[d] - p.ext_lo[d] for d in range(3)])) for lv in H.levels for p in lv)
    assert len(raw) == off + 2 * 24 * 8 * npatch
    ck = io.read_checkpoint(prefix)
    H2 = io.hierarchy_from_checkpoint(ck, seed=4, block_min=14, block_max=28)
    assert [(b.org, b.ex) for b in H2.blocks] == [(b.org, b.ex) for b in H.blocks]
    got = {}
    for lev, pid, back, data in io.checkpoint_patches(ck, H2):
        io.scatter_patch(H2, lev, pid, data, lambda bi, a: got.__setitem__((bi, back), a))
    for bi in range(len(H.blocks)):
        assert np.array_equal(got[(bi, 0)], cur[bi]) and np.array_equal(got[(bi, 1)], old[bi])
