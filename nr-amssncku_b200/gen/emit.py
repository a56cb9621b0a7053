"""Writes csrc/rhs_vjp_gen.cuh from the recorded tapes (see tape.py).

    make            (traces with trace_rhs.cpp, then runs this script)
"""
import os

import tape as TP

HERE = os.path.dirname(os.path.abspath(__file__))
HDR = """// rhs_vjp_gen.cuh -- GENERATED by gen/emit.py from gen/tape_*.txt; do not edit.
//
// Vector-Jacobian products recorded from the kernels' own point functions by
// gen/trace_rhs.cpp:
//   rhs_vjp_bssn / rhs_vjp_z4c: the pointwise right-hand side of the split
//     form (bssn_rhs_point with every stencil term an input);
//   ham_vjp / ham_fwd: the Hamiltonian constraint from the same inputs;
//   enforce_vjp: enforce_ga_point (in.c(0..5) metric offsets, 6..11 A~_ij).
// Inputs: centre values in.c(F) and D slots in.d(s) at the linearization
// point, output adjoints in.rb(F).  Outputs: out.cb(F, x), out.db(s, x), the
// adjoints of every input the outputs depend on.
#pragma once

namespace amss {

"""


def generate():
    """The text of csrc/rhs_vjp_gen.cuh from the tapes."""
    parts = [HDR]
    for name, fn in (("rhs_vjp_bssn", "tape_bssn.txt"), ("rhs_vjp_z4c", "tape_z4c.txt"),
                     ("ham_vjp", "tape_ham.txt"), ("enforce_vjp", "tape_enforce.txt")):
        tp = TP.Tape(os.path.join(HERE, fn))
        parts.append(TP.emit_vjp(tp, name))
        parts.append("\n")
    parts.append(TP.emit_fwd(TP.Tape(os.path.join(HERE, "tape_ham.txt")), "ham_fwd", 99))
    parts.append("\n")
    parts.append("}  // namespace amss\n")
    return "".join(parts)


def main():
    with open(os.path.join(HERE, "..", "csrc", "rhs_vjp_gen.cuh"), "w") as fh:
        fh.write(generate())


if __name__ == "__main__":
    main()
