// trace_rhs.cpp -- records the pointwise right-hand side of the split form as a
// straight-line program, for the adjoint generator (emit_vjp.py).
//
// The kernel's own point function (bssn_rhs_point in csrc/bssn_rhs.cuh, the
// path of the split form where every stencil term is an input) is compiled
// for the host with a recording scalar type `Rec`: every +, -, *, / it
// performs appends one node to a tape.  Inputs are the 24 (25) centre values
// and the D slots of the stencil pass; outputs are the right-hand sides and
// nothing more (each right-hand side's last operation adds its "adv" slot,
// upwinded advection + KO, itself an input).  The tape is printed as
//   N <count>
//   <id> in c <field>        centre value of a field
//   <id> in d <slot>         D slot
//   <id> k <value>           constant (hex float)
//   <id> <op> <a> <b>        + - * / ; n negate (b unused); p power (b: constant exponent)
//   out <field> <id>
// so the generated adjoint differentiates exactly what the forward computes.
#include <cmath>
#include <cstdio>
#include <map>
#include <vector>

#define AMSS_HOST_TRACE 1

namespace trace {
struct Node {
  char op;     // 'c' centre input, 'd' D input, 'k' constant, '+', '-', '*', '/', 'n' negate
  int a, b;    // operands (node ids) or input index
  double v;    // constant value
};
std::vector<Node> tape;
std::map<double, int> consts;
int push(char op, int a, int b, double v = 0.0) {
  tape.push_back(Node{op, a, b, v});
  return (int)tape.size() - 1;
}
int konst(double v) {
  auto it = consts.find(v);
  if (it != consts.end()) return it->second;
  const int id = push('k', -1, -1, v);
  consts[v] = id;
  return id;
}
}  // namespace trace

struct Rec {
  int id;
  Rec() : id(-1) {}
  Rec(double v) : id(trace::konst(v)) {}
  static Rec of(int i) {
    Rec r;
    r.id = i;
    return r;
  }
};
inline Rec operator+(Rec a, Rec b) { return Rec::of(trace::push('+', a.id, b.id)); }
inline Rec operator-(Rec a, Rec b) { return Rec::of(trace::push('-', a.id, b.id)); }
inline Rec operator*(Rec a, Rec b) { return Rec::of(trace::push('*', a.id, b.id)); }
inline Rec operator/(Rec a, Rec b) { return Rec::of(trace::push('/', a.id, b.id)); }
inline Rec operator-(Rec a) { return Rec::of(trace::push('n', a.id, -1)); }
inline Rec operator+(Rec a, double b) { return a + Rec(b); }
inline Rec operator+(double a, Rec b) { return Rec(a) + b; }
inline Rec operator-(Rec a, double b) { return a - Rec(b); }
inline Rec operator-(double a, Rec b) { return Rec(a) - b; }
inline Rec operator*(Rec a, double b) { return a * Rec(b); }
inline Rec operator*(double a, Rec b) { return Rec(a) * b; }
inline Rec operator/(Rec a, double b) { return a / Rec(b); }
inline Rec operator/(double a, Rec b) { return Rec(a) / b; }
// the NaN / inf screen of the point function does not enter the values
inline bool operator!=(Rec, Rec) { return false; }
inline bool operator>(Rec, Rec) { return false; }
inline bool operator<(Rec, Rec) { return false; }
inline bool isinf(Rec) { return false; }
// x^c for a constant exponent c (enforce_ga's det^(1/3))
inline Rec pow(Rec x, double c) { return Rec::of(trace::push('p', x.id, trace::konst(c))); }

#include "../csrc/bssn_step.cuh"

namespace amss {
template <>
struct wide<Rec> {
  using type = Rec;
};
}  // namespace amss

using namespace amss;

// Accessor: centre values and D slots are tape inputs.
struct RecPt {
  static constexpr bool kPre = true;
  using elem = Rec;
  long long p = 0;
  int i = 0, j = 0, k = 0;
  mutable std::map<int, int> cin, din;
  template <typename U, int F>
  U v(int, int, int) const {
    auto it = cin.find(F);
    if (it == cin.end()) it = cin.emplace(F, trace::push('c', F, -1)).first;
    return Rec::of(it->second);
  }
  template <typename U>
  U dv(int slot) const {
    auto it = din.find(slot);
    if (it == din.end()) it = din.emplace(slot, trace::push('d', slot, -1)).first;
    return Rec::of(it->second);
  }
};

struct RecEpi {
  std::map<int, int>* out;
  template <int F>
  void put(Rec v) {
    (*out)[F] = v.id;
  }
  void finish() {}
};

// Records only the Hamiltonian constraint (as output "field" 99).
struct RecHamEpi {
  std::map<int, int>* out;
  template <int F>
  void put(Rec) {}
  void finish() {}
  void ham(Rec v) { (*out)[99] = v.id; }
};

int main(int argc, char** argv) {
  // argument: "bssn" (default), "z4c", "ham" (the Hamiltonian constraint) or
  // "enforce" (enforce_ga_point)
  const char mode = argc > 1 ? argv[1][0] : 'b';
  RecPt q;
  Coefs<Rec> C{};
  PointGates G{};
  G.ord = 2;
  RhsAux aux{};
  std::map<int, int> out;
  if (mode == 'e') {
    // enforce_ga_point: inputs c0..c5 = the metric offsets, c6..c11 = A~_ij
    Rec gv[6], av[6];
    for (int m = 0; m < 6; ++m) {
      gv[m] = Rec::of(trace::push('c', m, -1));
      av[m] = Rec::of(trace::push('c', 6 + m, -1));
    }
    enforce_ga_point(gv, av);
    for (int m = 0; m < 6; ++m) {
      out[m] = gv[m].id;
      out[6 + m] = av[m].id;
    }
  } else if (mode == 'h') {
    RecHamEpi epi{&out};
    bssn_rhs_point<Rec, Rec, false, false, false>(q, C, G, aux, epi);
  } else {
    RecEpi epi{&out};
    if (mode == 'z')
      bssn_rhs_point<Rec, Rec, false, false, true>(q, C, G, aux, epi);
    else
      bssn_rhs_point<Rec, Rec, false, false, false>(q, C, G, aux, epi);
  }
  // each right-hand side ends by adding its "adv" slot (advection + KO): the
  // slot is an input like the others, so its adjoint is the output's
  std::printf("N %zu\n", trace::tape.size());
  for (size_t n = 0; n < trace::tape.size(); ++n) {
    const trace::Node& t = trace::tape[n];
    if (t.op == 'c') std::printf("%zu in c %d\n", n, t.a);
    else if (t.op == 'd') std::printf("%zu in d %d\n", n, t.a);
    else if (t.op == 'k') std::printf("%zu k %a\n", n, t.v);
    else std::printf("%zu %c %d %d\n", n, t.op, t.a, t.b);
  }
  for (auto& kv : out) std::printf("out %d %d\n", kv.first, kv.second);
  return 0;
}
