"""Checkpoint and resume through the reference's checkpoint format
(amss_b200.io.save_engine / load_engine, checkpoint::writecheck_cgh layout):
a run stopped after two coarse steps and resumed from its checkpoint takes the
next coarse step bit for bit like the run that never stopped (the resumed
engine needs the previous time levels and the level clocks for the time
interpolation of the children); dumps of an engine level hold its state."""
import numpy as np
import pytest

import amss_b200
from amss_b200 import io
from amss_b200.hierarchy import box_in_box
from amss_b200.regrid import Regridder
import amr as OA

pytestmark = pytest.mark.gpu
POS = [[1.2, 0.3, -0.4]]


def test_checkpoint_resume_is_bit_identical(tmp_path):
    H = box_in_box(40, 10.0, [tuple(POS[0])], 3, box_cells=32, seed=4, block_min=14, block_max=28)
    init = OA.initial_state(H, [1.0], POS, noise=1e-8)
    dt0 = 0.25 * H.h0
    e = amss_b200.Engine.from_hierarchy(H, precision="fp64", eps=0.1)
    for i, st in enumerate(init):
        e.set_state(i, st)
    for _ in range(2):
        e.coarse_step(dt0)
    assert e.sync() == 0
    prefix = str(tmp_path / "bssn")
    io.save_engine(prefix, e, H, Regridder(H, POS), 2 * dt0, dt0)
    e2, H2, t, r = io.load_engine(prefix, dt0, seed=4, block_min=14, block_max=28, precision="fp64", eps=0.1)
    assert t == 2 * dt0 and len(H2.blocks) == len(H.blocks)
    for lv in range(3):
        assert e2.level_steps(lv) == e.level_steps(lv)
    e.coarse_step(dt0)
    e2.coarse_step(dt0)
    assert e.sync() == 0 and e2.sync() == 0
    for i in range(len(H.blocks)):
        assert np.array_equal(e.get_state(i), e2.get_state(i))
        assert np.array_equal(e.get_time_level(i, 1), e2.get_time_level(i, 1))
    files = io.write_dump(str(tmp_path / "dump"), H, 2, 3 * dt0, dt0 / 4, lambda bi: e.get_state(bi), fields=[0])
    d = io.read_dump(files[0])
    want = io.patch_array(H, 2, 0, lambda bi: e.get_state(bi))[0]
    assert np.array_equal(d["data"], want)
    e.close()
    e2.close()
