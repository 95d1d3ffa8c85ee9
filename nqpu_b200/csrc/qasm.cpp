// OpenQASM 2.0 import and export of circuits.
//
// Follows the reference's OpenQASM 2.0 subset (circuits/formats/qasm.rs:65-362:
// `parse_qasm`, `execute_qasm`; export :363-510): `qreg`/`creg` declarations
// concatenated in declaration order, gate statements `name(params) args;`,
// `measure q[i] -> c[j];` and `measure q -> c;`, `//` comments, `OPENQASM` and
// `include` lines skipped.  Differences, all toward the OpenQASM 2.0 standard:
//   * parameters are expressions (numbers, pi, + - * / ^, unary minus,
//     parentheses), not only plain numbers (the reference reads "pi/2" as 0);
//   * the qelib1.inc gate set is mapped onto the engine's gates (u1/u2/u3/u,
//     sdg/tdg/sxdg, cy/ch/cu1/cu3, ccx/cswap, rzz/rxx/ryy, ...); an unknown
//     gate is an error instead of being skipped silently;
//   * a single-qubit gate applied to a whole register acts on every qubit of
//     it, two-qubit gates on two registers act pairwise;
//   * statements may span lines and several may share a line.
// `measure` becomes a measurement gate per qubit and `reset` a reset gate
// (mid-circuit: nqpu_circuit_execute_measured returns the outcomes in order,
// as the reference's execute_qasm collects measure_qubit results,
// qasm.rs:270-276); the classical bit a measurement writes is not tracked.
// `barrier` and `id` are no-ops.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/nqpu_b200.h"
#include "engine.h"
#include "planner.h"

namespace nqpu {
namespace {

constexpr double kPi = 3.14159265358979323846;

struct Reg {
  int base = 0, size = 0;
};

struct Parser {
  const std::string& src;
  size_t pos = 0;
  int line = 1;
  std::string err;
  int err_line = 0;
  std::map<std::string, Reg> qregs, cregs;
  int nq = 0, nc = 0;
  std::vector<GateRec> gates;
  std::vector<int> measured;

  explicit Parser(const std::string& s) : src(s) {}

  bool fail(const std::string& m) {
    if (err.empty()) {
      err = m;
      err_line = line;
    }
    return false;
  }
  void skip_ws() {
    while (pos < src.size()) {
      const char c = src[pos];
      if (c == '\n') {
        ++line;
        ++pos;
      } else if (std::isspace(static_cast<unsigned char>(c))) {
        ++pos;
      } else if (c == '/' && pos + 1 < src.size() && src[pos + 1] == '/') {
        while (pos < src.size() && src[pos] != '\n') ++pos;
      } else {
        break;
      }
    }
  }
  bool peek(char c) {
    skip_ws();
    return pos < src.size() && src[pos] == c;
  }
  bool accept(char c) {
    if (!peek(c)) return false;
    ++pos;
    return true;
  }
  bool expect(char c) {
    if (accept(c)) return true;
    return fail(std::string("expected '") + c + "'");
  }
  std::string ident() {
    skip_ws();
    const size_t b = pos;
    while (pos < src.size() && (std::isalnum(static_cast<unsigned char>(src[pos])) || src[pos] == '_')) ++pos;
    return src.substr(b, pos - b);
  }
  bool integer(int* out) {
    skip_ws();
    const size_t b = pos;
    while (pos < src.size() && std::isdigit(static_cast<unsigned char>(src[pos]))) ++pos;
    if (b == pos) return fail("expected an integer");
    const std::string s = src.substr(b, pos - b);
    if (s.size() > 9) return fail("integer out of range");
    *out = std::stoi(s);
    return true;
  }
  // expression grammar: sum := term (('+'|'-') term)*; term := unary (('*'|'/') unary)*;
  // unary := '-' unary | power; power := atom ('^' unary)?; atom := number | pi | '(' sum ')'
  bool expr(double* v) { return sum(v); }
  bool sum(double* v) {
    if (!term(v)) return false;
    for (;;) {
      if (accept('+')) {
        double r;
        if (!term(&r)) return false;
        *v += r;
      } else if (accept('-')) {
        double r;
        if (!term(&r)) return false;
        *v -= r;
      } else {
        return true;
      }
    }
  }
  bool term(double* v) {
    if (!unary(v)) return false;
    for (;;) {
      if (accept('*')) {
        double r;
        if (!unary(&r)) return false;
        *v *= r;
      } else if (accept('/')) {
        double r;
        if (!unary(&r)) return false;
        if (r == 0.0) return fail("division by zero in a parameter");
        *v /= r;
      } else {
        return true;
      }
    }
  }
  bool unary(double* v) {
    if (accept('-')) {
      if (!unary(v)) return false;
      *v = -*v;
      return true;
    }
    if (accept('+')) return unary(v);
    if (!atom(v)) return false;
    if (accept('^')) {
      double e;
      if (!unary(&e)) return false;
      *v = std::pow(*v, e);
    }
    return true;
  }
  bool atom(double* v) {
    skip_ws();
    if (accept('(')) {
      if (!sum(v)) return false;
      return expect(')');
    }
    if (pos < src.size() && (std::isdigit(static_cast<unsigned char>(src[pos])) || src[pos] == '.')) {
      const char* b = src.c_str() + pos;
      char* e = nullptr;
      *v = std::strtod(b, &e);
      if (e == b) return fail("bad number");
      pos += size_t(e - b);
      return true;
    }
    const std::string id = ident();
    if (id == "pi") {
      *v = kPi;
      return true;
    }
    return fail(id.empty() ? "expected a parameter" : "unknown symbol '" + id + "' in a parameter");
  }
  // argument: reg or reg[i]; returns the qubit list (whole register or one)
  bool qarg(std::vector<int>* out, bool classical = false) {
    const std::string name = ident();
    if (name.empty()) return fail("expected a register name");
    const auto& regs = classical ? cregs : qregs;
    auto it = regs.find(name);
    if (it == regs.end()) return fail("undeclared register '" + name + "'");
    out->clear();
    if (accept('[')) {
      int i;
      if (!integer(&i)) return false;
      if (!expect(']')) return false;
      if (i >= it->second.size) return fail("index out of range for register '" + name + "'");
      out->push_back(it->second.base + i);
    } else {
      for (int i = 0; i < it->second.size; ++i) out->push_back(it->second.base + i);
    }
    return true;
  }

  bool add(uint8_t code, const std::vector<int>& q, double p0 = 0, double p1 = 0, double p2 = 0, double p3 = 0) {
    GateRec g;
    g.code = code;
    g.nq = uint8_t(gate_arity(code));
    for (int i = 0; i < g.nq; ++i) g.q[i] = q[size_t(i)];
    for (int i = 0; i < g.nq; ++i)
      for (int j = i + 1; j < g.nq; ++j)
        if (g.q[i] == g.q[j]) return fail("a gate uses the same qubit twice");
    g.p[0] = p0;
    g.p[1] = p1;
    g.p[2] = p2;
    g.p[3] = p3;
    for (double x : g.p)
      if (!std::isfinite(x)) return fail("non-finite parameter");
    gates.push_back(g);
    return true;
  }
  bool add_custom1(const std::vector<int>& q, const cplx* m) {
    GateRec g;
    g.code = G_CUSTOM1;
    g.nq = 1;
    g.q[0] = q[0];
    for (int i = 0; i < 4; ++i) g.m[i] = m[i];
    gates.push_back(g);
    return true;
  }

  // one gate application on resolved qubit arguments (one qubit per argument)
  bool apply(const std::string& name, const std::vector<double>& p, const std::vector<int>& q) {
    auto need = [&](size_t np, size_t nqb) {
      if (p.size() != np) return fail("gate '" + name + "' takes " + std::to_string(np) + " parameters");
      if (q.size() != nqb) return fail("gate '" + name + "' takes " + std::to_string(nqb) + " qubits");
      return true;
    };
    const double P = kPi;
    if (name == "id" || name == "u0") return need(name == "u0" ? 1 : 0, 1);
    if (name == "h") return need(0, 1) && add(G_H, q);
    if (name == "x") return need(0, 1) && add(G_X, q);
    if (name == "y") return need(0, 1) && add(G_Y, q);
    if (name == "z") return need(0, 1) && add(G_Z, q);
    if (name == "s") return need(0, 1) && add(G_S, q);
    if (name == "t") return need(0, 1) && add(G_T, q);
    if (name == "sdg") return need(0, 1) && add(G_P, q, -P / 2);
    if (name == "tdg") return need(0, 1) && add(G_P, q, -P / 4);
    if (name == "sx") return need(0, 1) && add(G_SX, q);
    if (name == "sxdg") {
      if (!need(0, 1)) return false;
      const cplx m[4] = {cplx(0.5, -0.5), cplx(0.5, 0.5), cplx(0.5, 0.5), cplx(0.5, -0.5)};
      return add_custom1(q, m);
    }
    if (name == "rx") return need(1, 1) && add(G_RX, q, p[0]);
    if (name == "ry") return need(1, 1) && add(G_RY, q, p[0]);
    if (name == "rz") return need(1, 1) && add(G_RZ, q, p[0]);
    if (name == "p" || name == "u1") return need(1, 1) && add(G_P, q, p[0]);
    if (name == "u2") return need(2, 1) && add(G_U3, q, P / 2, p[0], p[1]);
    if (name == "u3" || name == "u" || name == "U") return need(3, 1) && add(G_U3, q, p[0], p[1], p[2]);
    if (name == "cx" || name == "CX") return need(0, 2) && add(G_CX, q);
    if (name == "cz") return need(0, 2) && add(G_CZ, q);
    if (name == "cy") return need(0, 2) && add(G_CU, q, P, P / 2, P / 2, 0);   // controlled U3(pi, pi/2, pi/2) = Y
    if (name == "ch") return need(0, 2) && add(G_CU, q, P / 2, 0, P, 0);        // controlled U3(pi/2, 0, pi) = H
    if (name == "swap") return need(0, 2) && add(G_SWAP, q);
    if (name == "iswap") return need(0, 2) && add(G_ISWAP, q);
    if (name == "cp" || name == "cu1" || name == "cphase") return need(1, 2) && add(G_CP, q, p[0]);
    if (name == "crx") return need(1, 2) && add(G_CRX, q, p[0]);
    if (name == "cry") return need(1, 2) && add(G_CRY, q, p[0]);
    if (name == "crz") return need(1, 2) && add(G_CRZ, q, p[0]);
    if (name == "cu3") return need(3, 2) && add(G_CU, q, p[0], p[1], p[2], 0);
    if (name == "cu") return need(4, 2) && add(G_CU, q, p[0], p[1], p[2], p[3]);
    if (name == "rzz") return need(1, 2) && add(G_RZZ, q, p[0]);
    if (name == "rxx") return need(1, 2) && add(G_RXX, q, p[0]);
    if (name == "ryy") return need(1, 2) && add(G_RYY, q, p[0]);
    if (name == "ccx") return need(0, 3) && add(G_CCX, q);
    if (name == "ccz") return need(0, 3) && add(G_CCZ, q);
    if (name == "cswap") return need(0, 3) && add(G_CSWAP, q);
    return fail("unknown gate '" + name + "'");
  }

  bool declaration(bool quantum) {
    const std::string name = ident();
    if (name.empty()) return fail("expected a register name");
    int size;
    if (!expect('[') || !integer(&size) || !expect(']') || !expect(';')) return false;
    auto& regs = quantum ? qregs : cregs;
    if (regs.count(name)) return fail("register '" + name + "' declared twice");
    int& counter = quantum ? nq : nc;
    regs[name] = Reg{counter, size};
    counter += size;
    if (quantum && nq > kMaxQubits) return fail("more than 34 qubits");
    return true;
  }

  bool statement() {
    const std::string kw = ident();
    if (kw.empty()) return fail("expected a statement");
    if (kw == "OPENQASM") {
      while (pos < src.size() && src[pos] != ';') ++pos;
      return expect(';');
    }
    if (kw == "include") {
      while (pos < src.size() && src[pos] != ';') {
        if (src[pos] == '\n') ++line;
        ++pos;
      }
      return expect(';');
    }
    if (kw == "qreg") return declaration(true);
    if (kw == "creg") return declaration(false);
    if (kw == "barrier") {
      while (pos < src.size() && src[pos] != ';') {
        if (src[pos] == '\n') ++line;
        ++pos;
      }
      return expect(';');
    }
    if (kw == "measure") {
      std::vector<int> q, c;
      if (!qarg(&q)) return false;
      skip_ws();
      if (src.compare(pos, 2, "->") != 0) return fail("expected '->'");
      pos += 2;
      if (!qarg(&c, true) || !expect(';')) return false;
      if (q.size() != c.size()) return fail("measure: register sizes differ");
      for (int x : q) {
        measured.push_back(x);
        if (!add(G_MEASURE, std::vector<int>{x})) return false;
      }
      return true;
    }
    if (kw == "reset") {
      std::vector<int> q;
      if (!qarg(&q) || !expect(';')) return false;
      for (int x : q)
        if (!add(G_RESET, std::vector<int>{x})) return false;
      return true;
    }
    if (kw == "gate" || kw == "opaque" || kw == "if")
      return fail("'" + kw + "' is not supported");
    // gate application
    std::vector<double> params;
    if (accept('(')) {
      if (!accept(')')) {
        for (;;) {
          double v;
          if (!expr(&v)) return false;
          params.push_back(v);
          if (accept(')')) break;
          if (!expect(',')) return false;
        }
      }
    }
    std::vector<std::vector<int>> args;
    for (;;) {
      std::vector<int> a;
      if (!qarg(&a)) return false;
      args.push_back(a);
      if (accept(';')) break;
      if (!expect(',')) return false;
    }
    // broadcast over whole-register arguments (all of the same length)
    size_t len = 1;
    for (const auto& a : args)
      if (a.size() != 1) {
        if (len != 1 && a.size() != len) return fail("register arguments of different sizes");
        len = a.size();
      }
    for (size_t i = 0; i < len; ++i) {
      std::vector<int> q;
      for (const auto& a : args) q.push_back(a.size() == 1 ? a[0] : a[i]);
      if (!apply(kw, params, q)) return false;
    }
    return true;
  }

  bool run() {
    for (;;) {
      skip_ws();
      if (pos >= src.size()) return true;
      if (!statement()) return false;
    }
  }
};

// OpenQASM text of one gate; false when the gate has no OpenQASM 2.0 form.
bool gate_qasm(const GateRec& g, std::ostringstream& o) {
  auto q = [&](int i) { return "q[" + std::to_string(g.q[i]) + "]"; };
  auto f = [&](double x) {
    std::ostringstream s;
    s.precision(17);
    s << x;
    return s.str();
  };
  switch (g.code) {
    case G_H: o << "h " << q(0); break;
    case G_X: o << "x " << q(0); break;
    case G_Y: o << "y " << q(0); break;
    case G_Z: o << "z " << q(0); break;
    case G_S: o << "s " << q(0); break;
    case G_T: o << "t " << q(0); break;
    case G_SX: o << "sx " << q(0); break;
    case G_RX: o << "rx(" << f(g.p[0]) << ") " << q(0); break;
    case G_RY: o << "ry(" << f(g.p[0]) << ") " << q(0); break;
    case G_RZ: o << "rz(" << f(g.p[0]) << ") " << q(0); break;
    case G_P: o << "p(" << f(g.p[0]) << ") " << q(0); break;
    case G_U3: o << "u3(" << f(g.p[0]) << "," << f(g.p[1]) << "," << f(g.p[2]) << ") " << q(0); break;
    case G_CX: o << "cx " << q(0) << "," << q(1); break;
    case G_CZ: o << "cz " << q(0) << "," << q(1); break;
    case G_SWAP: o << "swap " << q(0) << "," << q(1); break;
    case G_ISWAP: o << "iswap " << q(0) << "," << q(1); break;
    case G_CP: o << "cp(" << f(g.p[0]) << ") " << q(0) << "," << q(1); break;
    case G_CRX: o << "crx(" << f(g.p[0]) << ") " << q(0) << "," << q(1); break;
    case G_CRY: o << "cry(" << f(g.p[0]) << ") " << q(0) << "," << q(1); break;
    case G_CRZ: o << "crz(" << f(g.p[0]) << ") " << q(0) << "," << q(1); break;
    case G_RZZ: o << "rzz(" << f(g.p[0]) << ") " << q(0) << "," << q(1); break;
    case G_RXX: o << "rxx(" << f(g.p[0]) << ") " << q(0) << "," << q(1); break;
    case G_RYY: o << "ryy(" << f(g.p[0]) << ") " << q(0) << "," << q(1); break;
    case G_CCX: o << "ccx " << q(0) << "," << q(1) << "," << q(2); break;
    case G_CCZ: o << "ccz " << q(0) << "," << q(1) << "," << q(2); break;
    case G_CSWAP: o << "cswap " << q(0) << "," << q(1) << "," << q(2); break;
    case G_CU:
      o << "cu(" << f(g.p[0]) << "," << f(g.p[1]) << "," << f(g.p[2]) << "," << f(g.p[3]) << ") " << q(0) << ","
        << q(1);
      break;
    case G_MEASURE: o << "measure " << q(0) << " -> c[" << g.q[0] << "]"; break;
    case G_RESET: o << "reset " << q(0); break;
    default:
      o << "// gate code " << int(g.code) << " (custom matrix) has no OpenQASM 2.0 form";
      return false;
  }
  o << ";";
  return true;
}

}  // namespace
}  // namespace nqpu

using namespace nqpu;

extern "C" NqpuCircuit* nqpu_circuit_from_qasm(const char* text, uint32_t* error_line) {
  if (error_line) *error_line = 0;
  if (!text) return nullptr;
  const std::string src(text);
  Parser p(src);
  const bool ok = p.run();
  if (!ok || p.nq == 0) {
    if (error_line) *error_line = uint32_t(ok ? 1 : std::max(1, p.err_line));
    return nullptr;
  }
  auto* c = new (std::nothrow) CircuitImpl();
  if (!c) return nullptr;
  c->n = uint32_t(p.nq);
  c->gates = std::move(p.gates);
  c->version = 1;
  return reinterpret_cast<NqpuCircuit*>(c);
}

extern "C" uint32_t nqpu_circuit_num_qubits(const NqpuCircuit* circuit) {
  return circuit ? reinterpret_cast<const CircuitImpl*>(circuit)->n : 0u;
}

extern "C" NqpuError nqpu_circuit_to_qasm(const NqpuCircuit* circuit, char* out, uint64_t len, uint64_t* needed) {
  if (!circuit) return NQPU_NULL_POINTER;
  const CircuitImpl* c = reinterpret_cast<const CircuitImpl*>(circuit);
  std::ostringstream o;
  o << "OPENQASM 2.0;\ninclude \"qelib1.inc\";\nqreg q[" << c->n << "];\n";
  if (circuit_has_mid(c->gates)) o << "creg c[" << c->n << "];\n";
  bool all = true;
  for (const GateRec& g : c->gates) {
    all = gate_qasm(g, o) && all;
    o << "\n";
  }
  const std::string s = o.str();
  if (needed) *needed = s.size();
  if (out && len > 0) {
    const size_t k = std::min<size_t>(s.size(), size_t(len - 1));
    std::memcpy(out, s.data(), k);
    out[k] = '\0';
  }
  return all ? NQPU_OK : NQPU_INVALID_PARAMETER;
}
