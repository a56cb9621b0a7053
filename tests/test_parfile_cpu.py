"""The parameter-file front end (amss_b200.parfile) on CPU: the reference's
line grammar (misc::parse_parts, misc.C:71-196) and a par file written by the
reference's own generators for the amr workload (tests/golden/amr_workload.par,
made by tests/golden/make_parfile.py), which must give exactly the hierarchy,
time step, dissipation and punctures the bench builds by hand."""
import os

import pytest

from amss_b200 import parfile
from amss_b200.hierarchy import box_in_box

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "amr_workload.par")


def test_parse_line_follows_parse_parts():
    assert parfile.parse_line("   # only a comment") is None
    assert parfile.parse_line("") is None
    assert parfile.parse_line("ABE::Courant      = 0.25  # trailing") == ("ABE", "Courant", "0.25", (0, 0, 0))
    assert parfile.parse_line("  cgh::bbox[3][1][5]  = 6.0 ") == ("cgh", "bbox", "6.0", (3, 1, 5))
    assert parfile.parse_line("cgh::grids[4]       = 2") == ("cgh", "grids", "2", (4, 0, 0))
    assert parfile.parse_line('ABE::output dir = "binary output"') == ("ABE", "output dir", "binary output", (0, 0, 0))
    # the key keeps leading blanks and loses trailing ones (rTrim only), the group loses leading ones (lTrim)
    assert parfile.parse_line("BSSN:: chitiny = 1e-5")[1] == " chitiny"
    with pytest.raises(parfile.ParError):
        parfile.parse_line("ABE Courant 0.25")
    # a later line overrides an earlier one, as the driver's reads assign in order
    p = parfile.ParFile("ABE::Courant = 0.5\nABE::Courant = 0.25\n")
    assert p.get("ABE", "Courant", conv=float) == 0.25


def test_reference_generated_par_file_gives_the_amr_workload():
    cfg = parfile.load(GOLDEN, seed=1, block_min=18, block_max=74)
    ref = box_in_box(96, 48.0, [(-3.0, 0.0, 0.0), (3.0, 0.0, 0.0)], 7, box_cells=48, seed=1,
                     block_min=18, block_max=74)
    H = cfg.hierarchy
    assert (H.x0, H.h0) == (ref.x0, ref.h0) == (-48.0, 1.0)
    assert [[(p.lo, p.hi, p.buffer) for p in lv] for lv in H.levels] == \
        [[(p.lo, p.hi, p.buffer) for p in lv] for lv in ref.levels]
    assert [(b.level, b.patch, b.own_lo, b.own_hi, b.org, b.ex) for b in H.blocks] == \
        [(b.level, b.patch, b.own_lo, b.own_hi, b.org, b.ex) for b in ref.blocks]
    assert len(H.levels) == 7 and len(H.blocks) == 20
    assert (cfg.symmetry, cfg.eps, cfg.courant, cfg.dt0, cfg.chitiny) == (0, 0.1, 0.25, 0.25, 1e-5)
    assert cfg.masses == [0.5, 0.5]
    assert cfg.positions == [[-3.0, 0.0, 0.0], [3.0, 0.0, 0.0]]
    assert all(v == 0.0 for p in cfg.momenta + cfg.spins for v in p)


def test_unsupported_settings_are_refused():
    text = open(GOLDEN).read()
    with pytest.raises(parfile.ParError, match="time refinement"):
        parfile.load(text.replace("time refinement start from level =  0", "time refinement start from level =  2"))
    with pytest.raises(parfile.ParError, match="ID Type"):
        parfile.load(text.replace("ABE::ID Type    = -1", "ABE::ID Type    = 0"))
    with pytest.raises(parfile.ParError, match="shape says"):
        parfile.load(text.replace("cgh::shape[4][1][0] = 48", "cgh::shape[4][1][0] = 50"))
