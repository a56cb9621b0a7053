"""The oracle's compute_rhs_bssn against the reference's Fortran text.

Every whole-array assignment of the GAUGE 0 path of bssn_rhs.f90:5-1184
(preprocessed with GAUGE 0, ABV 0; continuation lines joined; comments,
declarations, calls and I/O dropped) must appear in oracle/bssn_oracle.c as
a pointwise assignment to the same array with the same token sequence on the
right-hand side, in the Fortran's order.  Identifiers compare without case
(Fortran is case-insensitive), `a[p]` and the oracle's local aliases
(`double uxx = gupxx[p]`) are resolved to the array names, and numeric
literals compare by value.  The few Fortran statements the oracle states in
another form (the NaN sum, the grid spacings, the parity vectors) are listed
below with the reason.

Reads the reference source, so it is skipped where the reference tree is not
mounted.
"""
import os
import re

import pytest

REF = "/root/reference/amss-ncku-python/AMSS_NCKU_source/bssn_rhs.f90"
ORACLE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "bssn_oracle.c")
MACROS = {"GAUGE": 0, "ABV": 0}

# Fortran statements of the path that the oracle states differently, by design
EXEMPT = {
    "dx": "bssn_rhs.f90:110-113 NaN sum; the oracle tests the fields themselves "
          "(oracle_state_has_nan), and dX/dY/dZ = X(2) - X(1) index from 1",
    "dy": "grid spacing, X(2) - X(1) with 1-based indexing",
    "dz": "grid spacing, X(2) - X(1) with 1-based indexing",
    "pi": "dacos(-ONE): the oracle takes the same double from acos(-1.0)",
    "gont": "return code, returned by the oracle function",
}
EXEMPT_PREFIX = ("sss(", "aas(", "asa(", "saa(", "ass(", "sas(", "ssa(")   # parity vectors, passed as arguments
# pointwise scalars of the oracle standing for the Fortran's whole arrays
SCALARS = {"ff": "f", "fc": "f", "c": "chin1", "al": "alpn1", "K": "trK", "db": "div_beta", "h": "ham_Res",
           "bxx": "betaxx", "bxy": "betaxy", "bxz": "betaxz", "byx": "betayx", "byy": "betayy",
           "byz": "betayz", "bzx": "betazx", "bzy": "betazy", "bzz": "betazz"}


def _preprocess(lines):
    """#if/#elif/#else/#endif with the macros above; #define/#undef/#include dropped."""
    out, stack = [], []   # stack of (active, taken)
    for ln in lines:
        s = ln.strip()
        if s.startswith("#"):
            d = s[1:].strip()
            word = d.split()[0] if d else ""
            if word in ("if", "elif"):
                expr = d[len(word):].strip()
                for k, v in MACROS.items():
                    expr = re.sub(rf"\b{k}\b", str(v), expr)
                expr = expr.replace("||", " or ").replace("&&", " and ")
                val = bool(eval(expr, {}, {}))
                if word == "if":
                    parent = all(a for a, _ in stack)
                    stack.append((parent and val, val))
                else:
                    a, taken = stack.pop()
                    parent = all(x for x, _ in stack)
                    stack.append((parent and val and not taken, taken or val))
            elif word == "else":
                a, taken = stack.pop()
                parent = all(x for x, _ in stack)
                stack.append((parent and not taken, True))
            elif word == "endif":
                stack.pop()
            continue
        if all(a for a, _ in stack):
            out.append(ln)
    return out


def _fortran_statements(path):
    lines = open(path).read().splitlines()[4:1184]          # bssn_rhs.f90:5-1184
    lines = _preprocess(lines)
    stmts, cur = [], ""
    for ln in lines:
        ln = ln.split("!")[0].rstrip()                       # no strings hold '!' on this path
        if not ln.strip():
            continue
        part = ln.strip()
        if part.startswith("&"):
            part = part[1:]
        if part.endswith("&"):
            cur += part[:-1] + " "
            continue
        stmts.append(cur + part)
        cur = ""
    out = []
    for s in stmts:
        low = s.strip().lower()
        if "::" in low or low.startswith(("call ", "if", "endif", "end ", "do ", "enddo", "return", "subroutine",
                                          "implicit", "write", "else", "integer", "real", "double", "logical")):
            continue
        m = re.match(r"^\s*([A-Za-z_][A-Za-z0-9_]*(\([^=]*\))?)\s*=(?!=)(.*)$", s)
        if not m:
            continue
        out.append((m.group(1).replace(" ", "").lower(), m.group(3)))
    return out


def _expand_macros(body):
    """Expand the oracle's one-argument helper macros (#define NAME(a) ...)
    other than G(a), which _tokens resolves; drop the directives."""
    body = body.replace("\\\n", " ")
    defs = {}
    for m in re.finditer(r"^\s*#define\s+(\w+)\((\w+)\)\s+(.*)$", body, re.M):
        if m.group(1) != "G":
            defs[m.group(1)] = (m.group(2), m.group(3))
    body = re.sub(r"^\s*#.*$", " ", body, flags=re.M)
    for name, (arg, text) in defs.items():
        body = re.sub(rf"\b{name}\((\w+)\)", lambda mm: re.sub(rf"\b{arg}\b", mm.group(1), text), body)
    return body


def _c_statements(path):
    src = open(path).read()
    body = src[src.index("int oracle_compute_rhs_bssn("):]
    body = body[:body.index("\n}\n")]
    body = re.sub(r"/\*.*?\*/", " ", body, flags=re.S)
    body = re.sub(r"//[^\n]*", " ", body)
    body = _expand_macros(body)
    out, alias = [], {}
    for st in body.split(";"):
        st = st.strip()
        if not st:
            continue
        st = re.sub(r"\bPL\b", " ", st)
        st = st.replace("{", " ").replace("}", " ").strip()
        if st.startswith("if (") and ")" in st:
            st = st[st.index(")") + 1:].strip()
        m = re.match(r"^double\s+(.*)$", st, re.S)
        if m:
            for part in _split_top(m.group(1)):
                mm = re.match(r"^\s*(\w+)\s*=\s*(.*?)\s*$", part, re.S)
                if not mm:
                    continue
                name, expr = mm.group(1), mm.group(2)
                ma = re.match(r"^(\w+)\[p\]$", expr)
                if ma:                              # double uxx = gupxx[p]: an alias of the array
                    alias[name] = ma.group(1)
                elif name in SCALARS:
                    alias[name] = SCALARS[name]
                    if not re.match(r"^\w+$", expr):   # a pointwise value the Fortran keeps in an array
                        out.append((SCALARS[name].lower(), expr, dict(alias)))
            continue
        m = re.match(r"^(\w+)\[p\]\s*=(?!=)(.*)$", st, re.S)
        if m:
            out.append((m.group(1).lower(), m.group(2), dict(alias)))
            continue
        m = re.match(r"^(\w+)\s*=(?!=)(.*)$", st, re.S)
        if m and m.group(1) in SCALARS:
            out.append((SCALARS[m.group(1)].lower(), m.group(2), dict(alias)))
    return out


def _split_top(text):
    """Split a declarator list at the commas outside parentheses."""
    parts, depth, cur = [], 0, ""
    for ch in text:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return parts


TOKEN = re.compile(r"\d+\.\d*(?:[dDeE][+-]?\d+)?|\.\d+(?:[dDeE][+-]?\d+)?|\d+(?:[dDeE][+-]?\d+)?|\w+|\*\*|[-+*/()]")


def _tokens(expr, alias=None):
    expr = re.sub(r"\bG\((\w+)\)", r"\1", expr)
    expr = re.sub(r"(\w+)\[p\]", r"\1", expr)
    toks = []
    for t in TOKEN.findall(expr):
        if re.match(r"^[\d.]", t):
            toks.append(repr(float(t.lower().replace("d", "e"))))
        else:
            if alias and t in alias:
                t = alias[t]
            toks.append(t.lower().rstrip("_"))   # Gamyy_: the oracle's name for the Fortran's Gamyy
    return toks


@pytest.mark.skipif(not os.path.exists(REF), reason="reference source not mounted")
def test_oracle_statements_follow_the_fortran():
    fort = _fortran_statements(REF)
    cst = [(lhs, _tokens(rhs, al)) for lhs, rhs, al in _c_statements(ORACLE)]
    checked, missing, pos = 0, [], 0
    for lhs, rhs in fort:
        if lhs in EXEMPT or lhs.startswith(EXEMPT_PREFIX):
            continue
        want = _tokens(rhs)
        # the next oracle assignment to the same array with the same tokens, in order
        for q in range(pos, len(cst)):
            if cst[q][0] == lhs and cst[q][1] == want:
                pos = q + 1
                checked += 1
                break
        else:
            missing.append((lhs, " ".join(want)[:160]))
    assert not missing, f"{len(missing)} Fortran statements without their oracle twin: {missing[:6]}"
    assert checked >= 180, checked
