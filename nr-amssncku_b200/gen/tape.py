"""Straight-line programs recorded by trace_rhs.cpp: parsing, evaluation, and
the reverse-mode (VJP) code emitted from them.

A tape is a list of nodes in execution order: inputs (centre values 'c' of a
field, D slots 'd'), constants 'k', and binary/unary arithmetic ('+', '-',
'*', '/', 'n' negate), plus the node that holds each output field.
"""
import numpy as np


class Tape:
    def __init__(self, path):
        self.op, self.a, self.b, self.val = [], [], [], []
        self.inputs_c, self.inputs_d = {}, {}   # field / slot -> node
        self.outputs = {}                         # field -> node
        with open(path) as fh:
            n = int(fh.readline().split()[1])
            for _ in range(n):
                p = fh.readline().split()
                i = int(p[0])
                assert i == len(self.op)
                if p[1] == "in":
                    self.op.append(p[2])
                    self.a.append(int(p[3]))
                    self.b.append(-1)
                    self.val.append(0.0)
                    (self.inputs_c if p[2] == "c" else self.inputs_d)[int(p[3])] = i
                elif p[1] == "k":
                    self.op.append("k")
                    self.a.append(-1)
                    self.b.append(-1)
                    self.val.append(float.fromhex(p[2]))
                else:
                    self.op.append(p[1])
                    self.a.append(int(p[2]))
                    self.b.append(int(p[3]))
                    self.val.append(0.0)
            for line in fh:
                p = line.split()
                if p and p[0] == "out":
                    self.outputs[int(p[1])] = int(p[2])
        self.live = self._live()

    def _live(self):
        """Nodes an output depends on."""
        live = np.zeros(len(self.op), dtype=bool)
        stack = list(self.outputs.values())
        while stack:
            i = stack.pop()
            if live[i]:
                continue
            live[i] = True
            for j in (self.a[i], self.b[i]):
                if j >= 0 and self.op[i] not in ("c", "d", "k"):
                    stack.append(j)
        return live

    def evaluate(self, c, d):
        """Outputs {field: array} for centre values c[field] and D slots d[slot]
        (arrays of one shape)."""
        v = [None] * len(self.op)
        for i, op in enumerate(self.op):
            if not self.live[i]:
                continue
            if op == "c":
                v[i] = c[self.a[i]]
            elif op == "d":
                v[i] = d[self.a[i]]
            elif op == "k":
                v[i] = self.val[i]
            elif op == "+":
                v[i] = v[self.a[i]] + v[self.b[i]]
            elif op == "-":
                v[i] = v[self.a[i]] - v[self.b[i]]
            elif op == "*":
                v[i] = v[self.a[i]] * v[self.b[i]]
            elif op == "/":
                v[i] = v[self.a[i]] / v[self.b[i]]
            elif op == "n":
                v[i] = -v[self.a[i]]
            elif op == "p":
                v[i] = v[self.a[i]] ** v[self.b[i]]
            else:
                raise ValueError(op)
        return {f: v[i] for f, i in self.outputs.items()}


def vjp(tape, c, d, rb):
    """Reverse sweep in numpy: (cb {field: array}, db {slot: array}) for output
    adjoints rb[field] at the point (c, d) -- the same algorithm emit_vjp writes."""
    n = len(tape.op)
    v = [None] * n
    for i, op in enumerate(tape.op):
        if not tape.live[i]:
            continue
        if op == "c":
            v[i] = c[tape.a[i]]
        elif op == "d":
            v[i] = d[tape.a[i]]
        elif op == "k":
            v[i] = tape.val[i]
        elif op == "+":
            v[i] = v[tape.a[i]] + v[tape.b[i]]
        elif op == "-":
            v[i] = v[tape.a[i]] - v[tape.b[i]]
        elif op == "*":
            v[i] = v[tape.a[i]] * v[tape.b[i]]
        elif op == "/":
            v[i] = v[tape.a[i]] / v[tape.b[i]]
        elif op == "n":
            v[i] = -v[tape.a[i]]
        elif op == "p":
            v[i] = v[tape.a[i]] ** v[tape.b[i]]
    adj = [None] * n

    def add(j, x):
        if tape.op[j] == "k":
            return
        adj[j] = x if adj[j] is None else adj[j] + x

    for f, i in tape.outputs.items():
        add(i, rb[f])
    for i in range(n - 1, -1, -1):
        if not tape.live[i] or adj[i] is None or tape.op[i] in ("c", "d", "k"):
            continue
        op, a, b, g = tape.op[i], tape.a[i], tape.b[i], adj[i]
        if op == "+":
            add(a, g)
            add(b, g)
        elif op == "-":
            add(a, g)
            add(b, -g)
        elif op == "n":
            add(a, -g)
        elif op == "*":
            add(a, g * v[b])
            add(b, g * v[a])
        elif op == "/":
            add(a, g / v[b])
            add(b, -(g * v[i] / v[b]))
        elif op == "p":
            add(a, g * v[b] * v[i] / v[a])
    cb = {f: adj[i] for f, i in tape.inputs_c.items() if adj[i] is not None}
    db = {s: adj[i] for s, i in tape.inputs_d.items() if adj[i] is not None}
    return cb, db


def emit_vjp(tape, name):
    """CUDA source of `name`: the vector-Jacobian product of the tape.

    template <typename T, typename In, typename Out>
    __device__ void name(const In& in, Out& out)
      in.c(F), in.d(slot): the linearization point; in.rb(F): output adjoints;
      out.cb(F, value), out.db(slot, value): adjoints of the inputs (each
      called once per input the outputs depend on).
    """
    L = []
    w = L.append
    val = lambda i: (repr_k(tape.val[i]) if tape.op[i] == "k" else f"v{i}")
    w(f"template <typename T, typename In, typename Out>")
    w(f"__device__ __forceinline__ void {name}(const In& in, Out& out) {{")
    # forward sweep
    for i, op in enumerate(tape.op):
        if not tape.live[i] or op == "k":
            continue
        if op == "c":
            w(f"  const T v{i} = in.c({tape.a[i]});")
        elif op == "d":
            w(f"  const T v{i} = in.d({tape.a[i]});")
        elif op == "n":
            w(f"  const T v{i} = -{val(tape.a[i])};")
        elif op == "p":
            w(f"  const T v{i} = pow({val(tape.a[i])}, {val(tape.b[i])});")
        else:
            w(f"  const T v{i} = {val(tape.a[i])} {op} {val(tape.b[i])};")
    # reverse sweep
    defined = set()
    contrib = {}

    def add(j, expr, neg=False):
        if tape.op[j] == "k":
            return
        sign = "-" if neg else "+"
        if j in defined:
            w(f"  a{j} {sign}= {expr};")
        else:
            w(f"  T a{j} = {'-' if neg else ''}({expr});")
            defined.add(j)

    out_of = {}
    for f, i in tape.outputs.items():
        out_of.setdefault(i, []).append(f)
    for i in range(len(tape.op) - 1, -1, -1):
        if not tape.live[i]:
            continue
        for f in out_of.get(i, []):
            add(i, f"in.rb({f})")
        op = tape.op[i]
        if op in ("c", "d", "k") or i not in defined:
            continue
        a, b = tape.a[i], tape.b[i]
        if op == "+":
            add(a, f"a{i}")
            add(b, f"a{i}")
        elif op == "-":
            add(a, f"a{i}")
            add(b, f"a{i}", neg=True)
        elif op == "n":
            add(a, f"a{i}", neg=True)
        elif op == "*":
            add(a, f"a{i} * {val(b)}")
            add(b, f"a{i} * {val(a)}")
        elif op == "/":
            add(a, f"a{i} / {val(b)}")
            add(b, f"a{i} * v{i} / {val(b)}", neg=True)
        elif op == "p":
            add(a, f"a{i} * {val(b)} * v{i} / {val(a)}")
    for f, i in sorted(tape.inputs_c.items()):
        if i in defined:
            w(f"  out.cb({f}, a{i});")
    for s, i in sorted(tape.inputs_d.items()):
        if i in defined:
            w(f"  out.db({s}, a{i});")
    w("}")
    mask = sum(1 << f for f, i in tape.inputs_c.items() if i in defined)
    w(f"// centre fields whose adjoint {name} writes (bit F)")
    w(f"constexpr unsigned long long {name}_cb_mask = 0x{mask:x}ull;")
    return "\n".join(L) + "\n"


def emit_fwd(tape, name, field):
    """CUDA source of `name`: the tape's output `field` as a function of in.c /
    in.d (template <typename T, typename In> __device__ T name(const In& in))."""
    L = []
    w = L.append
    val = lambda i: (repr_k(tape.val[i]) if tape.op[i] == "k" else f"v{i}")
    w(f"template <typename T, typename In>")
    w(f"__device__ __forceinline__ T {name}(const In& in) {{")
    for i, op in enumerate(tape.op):
        if not tape.live[i] or op == "k":
            continue
        if op == "c":
            w(f"  const T v{i} = in.c({tape.a[i]});")
        elif op == "d":
            w(f"  const T v{i} = in.d({tape.a[i]});")
        elif op == "n":
            w(f"  const T v{i} = -{val(tape.a[i])};")
        elif op == "p":
            w(f"  const T v{i} = pow({val(tape.a[i])}, {val(tape.b[i])});")
        else:
            w(f"  const T v{i} = {val(tape.a[i])} {op} {val(tape.b[i])};")
    w(f"  return {val(tape.outputs[field])};")
    w("}")
    return "\n".join(L) + "\n"


def repr_k(x):
    return f"T({float(x).hex()})"
