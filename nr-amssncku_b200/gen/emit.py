"""Writes csrc/rhs_vjp_gen.cuh from the recorded tapes (see tape.py).

    python emit.py        (after: g++ -std=c++17 -O0 -o trace_rhs trace_rhs.cpp;
                                  ./trace_rhs > tape_bssn.txt; ./trace_rhs z > tape_z4c.txt)
"""
import os

import tape as TP

HERE = os.path.dirname(os.path.abspath(__file__))
HDR = """// rhs_vjp_gen.cuh -- GENERATED by gen/emit.py from gen/tape_{bssn,z4c}.txt; do not edit.
//
// Vector-Jacobian products of the pointwise right-hand side of the split form
// (bssn_rhs_point with every stencil term an input), recorded from the
// kernel's own point function by gen/trace_rhs.cpp.  Inputs: the 24 (25)
// centre values in.c(F) and the D slots in.d(s) at the linearization point,
// the output adjoints in.rb(F).  Outputs: out.cb(F, x), out.db(s, x), the
// adjoints of every input the right-hand side depends on.
#pragma once

namespace amss {

"""


def main():
    parts = [HDR]
    for name, fn in (("rhs_vjp_bssn", "tape_bssn.txt"), ("rhs_vjp_z4c", "tape_z4c.txt")):
        tp = TP.Tape(os.path.join(HERE, fn))
        parts.append(TP.emit_vjp(tp, name))
        parts.append("\n")
    parts.append("}  // namespace amss\n")
    with open(os.path.join(HERE, "..", "csrc", "rhs_vjp_gen.cuh"), "w") as fh:
        fh.write("".join(parts))


if __name__ == "__main__":
    main()
