"""The analysis output files of an evolution: bssn_constraint.dat from the
engine's constraint monitor, and bssn_psi4.dat from its wave extraction.

File format and cadence follow the reference:

* monitor::monitor (monitor.C:15-101): the file is <out_dir>/<name>; when it
  exists already (a run restarted from a checkpoint) the name becomes
  1_<name>, 2_<name>, ... (monitor.C:79-86).  Three header lines: "# File
  created on " + asctime() (which ends in a newline), "#", and the column
  header "# time Ham Px Py Pz Gx Gy Gz" (bssn_class.C:100-103).
* monitor::writefile (monitor.C:137-150): iostream with setprecision(8), the
  default float format (that is printf's %.8g) and ios::left set by the
  constructor: the time in a field of 14, then per value a blank and a field
  of 15, one line per call.
* bssn_class::Constraint_Out (bssn_class.C:7296-7300, 7472-7505): every call
  adds the coarse step dT * 0.5^max(0, trfls) to LastConsOut; once that reaches
  AnasTime, one line per level (levels in order, all at the same PhysTime) with
  the 7 norms of Parallel::L2Norm, and LastConsOut goes back to 0.  A Z4c run
  writes 8 values per line, Theta's norm last (Z4c_class.C:2502-2511).  The
  reference takes the norms over the first patch of each level
  (Parallel::L2Norm(GH->PatL[lev]->data, ...), bssn_class.C:7475), and so does
  ConstraintMonitor by default; first_patch=False sums every patch, which
  differs on levels of two or more patches.
* bssn_psi4.dat (bssn_class.C:76-88 header, :7143-7263 AnalysisStuff): the
  column header names R{l:02d}m{m:03d} and I{l:02d}m{m:03d} for l = 2..maxl,
  m = -l..l, each in a field of 16 after "# time" in a field of 15; one line
  per detector radius (maxrex, maxrex - drex, ...) with the time and the
  (RP, IP) pairs (monitor::writefile with two arrays, monitor.C:151-165);
  bssn_ADMQs.dat the same lines with the 7 ADM integrals of surf_MassPAng.
"""
import os
import time

HEADER = "# time Ham Px Py Pz Gx Gy Gz"


def format_line(t, values):
    """One monitor::writefile line (without the newline)."""
    return "%-14.8g" % t + "".join(" %-15.8g" % v for v in values)


def open_name(out_dir, name):
    """monitor.C:79-86: the first of name, 1_name, 2_name, ... that does not exist."""
    path = os.path.join(out_dir, name)
    i = 1
    while os.path.exists(path):
        path = os.path.join(out_dir, f"{i}_{name}")
        i += 1
    return path


class ConstraintMonitor:
    """bssn_constraint.dat for an engine.  `anas_time` is the output
    interval (AnasTime), `trfls` the level below which there is no time
    refinement (0 on the engine's hierarchies), `z4c` adds Theta's column."""

    def __init__(self, out_dir, anas_time, name="bssn_constraint.dat", trfls=0, z4c=False, first_patch=True):
        self.first_patch = first_patch
        self.path = open_name(out_dir, name)
        self.anas_time = float(anas_time)
        self.trfls = int(trfls)
        self.nvals = 8 if z4c else 7
        self.last = 0.0   # LastConsOut
        with open(self.path, "w") as f:
            f.write("# File created on " + time.asctime() + "\n")
            f.write("#\n")
            f.write(HEADER + "\n")

    def write(self, engine, phys_time, nlevels):
        """One line per level of the engine's current state at phys_time."""
        with open(self.path, "a") as f:
            for lv in range(nlevels):
                c = engine.constraint_norms(lv, first_patch=self.first_patch)
                f.write(format_line(phys_time, c[:self.nvals]) + "\n")

    def after_step(self, engine, phys_time, dT, nlevels):
        """Constraint_Out after a coarse step of dT ending at phys_time;
        returns True when it wrote."""
        self.last += dT * 0.5 ** max(0, self.trfls)
        if self.last >= self.anas_time:
            self.write(engine, phys_time, nlevels)
            self.last = 0.0
            return True
        return False


def psi4_header(maxl):
    """bssn_class.C:76-88: the column header of bssn_psi4.dat."""
    s = "%-15s" % "# time"
    for l in range(2, maxl + 1):
        for m in range(-l, l + 1):
            s += "%-16s" % ("R%02dm%03d" % (l, m)) + "%-16s" % ("I%02dm%03d" % (l, m))
    return s


ADM_HEADER = "%-15s" % "# time ADMmass ADMPx ADMPy ADMPz ADMSx ADMSy ADMSz"   # bssn_class.C:95-98


class WaveMonitor:
    """bssn_psi4.dat and bssn_ADMQs.dat for an engine: at each analysis
    time, Psi4 of level `level` and its modes, and the ADM mass, momentum and
    angular momentum, on decn spheres of radius maxrex, maxrex - drex, ...
    (AnalysisStuff, bssn_class.C:6945-7285, every AnasTime of the analysis
    level's clock)."""

    def __init__(self, out_dir, anas_time, level, maxl=8, decn=1, maxrex=None, drex=0.0, nquarter=40,
                 name="bssn_psi4.dat", adm_name="bssn_ADMQs.dat"):
        if maxrex is None:
            raise ValueError("WaveMonitor: maxrex (the outermost extraction radius) is required")
        self.path = open_name(out_dir, name)
        self.adm_path = open_name(out_dir, adm_name)
        self.anas_time = float(anas_time)
        self.level, self.maxl, self.decn = int(level), int(maxl), int(decn)
        self.maxrex, self.drex, self.nquarter = float(maxrex), float(drex), int(nquarter)
        self.last = 0.0   # LastAnas
        for path, head in ((self.path, psi4_header(self.maxl)), (self.adm_path, ADM_HEADER)):
            with open(path, "w") as f:
                f.write("# File created on " + time.asctime() + "\n")
                f.write("#\n")
                f.write(head + "\n")

    def write(self, engine, phys_time):
        engine.psi4(self.level)
        rex = self.maxrex
        with open(self.path, "a") as f, open(self.adm_path, "a") as g:
            for _ in range(self.decn):
                rp, ip = engine.psi4_modes(self.level, rex, self.nquarter, self.maxl)
                vals = [v for pair in zip(rp, ip) for v in pair]
                f.write(format_line(phys_time, vals) + "\n")
                g.write(format_line(phys_time, engine.adm_integrals(self.level, rex, self.nquarter)) + "\n")
                rex -= self.drex

    def after_step(self, engine, phys_time, dT_lev):
        """AnalysisStuff's clock: LastAnas += dT_lev; write when it reaches
        AnasTime.  Returns True when it wrote."""
        self.last += dT_lev
        if self.last >= self.anas_time:
            self.write(engine, phys_time)
            self.last = 0.0
            return True
        return False
