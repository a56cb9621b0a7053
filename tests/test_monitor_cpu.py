"""The constraint output file (amss_b200.monitor) on the CPU: the line format
against the iostream formatting monitor::writefile uses (monitor.C:137-150),
the restart naming (monitor.C:79-86) and the Constraint_Out cadence
(bssn_class.C:7296-7300) with a stand-in engine."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from amss_b200 import monitor

VALUES = [0.0, 0.25, 1.5e-7, 3.3752749694333035, 12345678.9, 1e-300, -2.5e10, 100.0, 0.1 + 0.2]

CPP = r"""
#include <iomanip>
#include <iostream>
int main() {
  const double v[] = {%s};
  std::cout.setf(std::ios::left);
  std::cout << std::setprecision(8);
  std::cout << std::setw(14) << %r;
  for (double x : v) std::cout << " " << std::setw(15) << x;
  std::cout << std::endl;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_line_matches_iostream(tmp_path):
    t = 12.375
    src = tmp_path / "fmt.cpp"
    src.write_text(CPP % (", ".join(repr(v) for v in VALUES), t))
    exe = tmp_path / "fmt"
    subprocess.run(["g++", "-O0", "-o", str(exe), str(src)], check=True)
    want = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.rstrip("\n")
    assert monitor.format_line(t, VALUES) == want


def test_restart_names(tmp_path):
    a = monitor.ConstraintMonitor(str(tmp_path), 1.0)
    b = monitor.ConstraintMonitor(str(tmp_path), 1.0)
    c = monitor.ConstraintMonitor(str(tmp_path), 1.0)
    assert [os.path.basename(m.path) for m in (a, b, c)] == \
        ["bssn_constraint.dat", "1_bssn_constraint.dat", "2_bssn_constraint.dat"]
    lines = open(a.path).read().splitlines()
    assert lines[0].startswith("# File created on ") and lines[1] == "#" and lines[2] == monitor.HEADER


class _FakeEngine:
    def __init__(self):
        self.calls = []

    def constraint_norms(self, level, first_patch=False):
        assert first_patch   # the monitor file takes the reference's first patch by default
        self.calls.append(level)
        return np.arange(8, dtype=float) + 10.0 * level + 0.5


@pytest.mark.parametrize("z4c", [False, True])
def test_cadence_and_levels(tmp_path, z4c):
    m = monitor.ConstraintMonitor(str(tmp_path), anas_time=1.0, z4c=z4c)
    eng = _FakeEngine()
    wrote = [m.after_step(eng, 0.25 * (s + 1), 0.25, nlevels=3) for s in range(8)]
    assert wrote == [False, False, False, True, False, False, False, True]
    assert eng.calls == [0, 1, 2, 0, 1, 2]
    rows = open(m.path).read().splitlines()[3:]
    assert len(rows) == 6
    for r, (t, lv) in zip(rows, [(1.0, 0), (1.0, 1), (1.0, 2), (2.0, 0), (2.0, 1), (2.0, 2)]):
        vals = [float(x) for x in r.split()]
        assert vals[0] == t
        assert vals[1:] == list(np.arange(8 if z4c else 7) + 10.0 * lv + 0.5)


class _FakeWaveEngine:
    def __init__(self):
        self.calls = []

    def psi4(self, level):
        self.calls.append(("psi4", level))

    def psi4_modes(self, level, rex, nquarter, maxl):
        self.calls.append(("modes", level, rex, nquarter, maxl))
        nn = (maxl + 1) ** 2 - 4
        return np.arange(nn) + rex, -(np.arange(nn) + rex)

    def adm_integrals(self, level, rex, nquarter):
        self.calls.append(("adm", level, rex, nquarter))
        return np.arange(7) * 0.5 + rex


def test_psi4_header_names_every_mode():
    """bssn_class.C:76-88: "# time" in a field of 15, then R%02dm%03d and
    I%02dm%03d in fields of 16 for l = 2..maxl, m = -l..l."""
    h = monitor.psi4_header(3)
    assert h.startswith("# time         R02m-02         I02m-02         R02m-01")
    names = h.split()[2:]
    assert len(names) == 2 * ((3 + 1) ** 2 - 4)
    assert names[-2:] == ["R03m003", "I03m003"]


def test_wave_monitor_radii_and_columns(tmp_path):
    """AnalysisStuff: every AnasTime of the analysis level's clock, Psi4 once,
    then per detector radius maxrex, maxrex - drex, ... one bssn_psi4.dat line
    of (RP, IP) pairs and one bssn_ADMQs.dat line of the 7 ADM integrals."""
    m = monitor.WaveMonitor(str(tmp_path), anas_time=0.5, level=2, maxl=2, decn=2, maxrex=40.0, drex=10.0, nquarter=6)
    eng = _FakeWaveEngine()
    wrote = [m.after_step(eng, 0.25 * (s + 1), 0.25) for s in range(4)]
    assert wrote == [False, True, False, True]
    assert eng.calls[:4] == [("psi4", 2), ("modes", 2, 40.0, 6, 2), ("adm", 2, 40.0, 6), ("modes", 2, 30.0, 6, 2)]
    rows = open(m.path).read().splitlines()
    assert rows[2] == monitor.psi4_header(2)
    vals = [float(x) for x in rows[3].split()]
    assert vals[0] == 0.5 and len(vals) == 1 + 2 * 5
    assert vals[1::2] == [40.0 + k for k in range(5)] and vals[2::2] == [-(40.0 + k) for k in range(5)]
    adm = open(m.adm_path).read().splitlines()
    assert adm[2] == "# time ADMmass ADMPx ADMPy ADMPz ADMSx ADMSy ADMSz"
    assert [float(x) for x in adm[4].split()] == [0.5] + list(np.arange(7) * 0.5 + 30.0)
    assert len(rows) == 3 + 4 and len(adm) == 3 + 4
