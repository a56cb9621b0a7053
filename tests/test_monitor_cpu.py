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
