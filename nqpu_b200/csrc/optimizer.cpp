// Circuit optimizer pre-pass (host, on the gate list).
//
// Restates the reference's CircuitOptimizer (circuits/synthesis/
// circuit_optimizer.rs:115-735) on this engine's gate records, with the same
// passes, order, levels and tolerances:
//   1. Clifford simplification (:250): adjacent identical self-inverse gates
//      (H, X, Y, Z, CNOT, CZ, SWAP) on the same targets and controls cancel;
//   2. peephole (:612, Aggressive): H(t) CX(c,t) H(t) -> CZ(c,t),
//      H(t) CZ(c,t) H(t) -> CX(c,t), CX(c,t) X(t) CX(c,t) -> X(t),
//      S S -> Z, T T -> S;
//   3. rotation merging (:424, Basic and up): Rx(a) Rx(b) -> Rx(a+b) (and Ry,
//      Rz), both dropped when |a+b| < 1e-10;
//   4. commutation analysis (:508, Moderate and up): up to five bubble passes
//      swapping adjacent commuting gates when that brings a gate next to one
//      it cancels or merges with;
//   5. gate fusion (:303, Basic and up): a run of >= 2 single-qubit gates on
//      one qubit becomes one custom 2x2 gate (product in circuit order), or
//      nothing when the product is the identity or a global phase (1e-10);
//   and a final Clifford simplification.
// Mid-circuit measurements and resets are never moved, merged or cancelled.
#include <cmath>
#include <complex>
#include <vector>

#include "../../include/nqpu_b200.h"
#include "engine.h"
#include "planner.h"

namespace nqpu {
namespace {

struct View {
  int targets[3];
  int nt = 0;
  int controls[3];
  int nc = 0;
};

View view(const GateRec& g) {
  View v;
  auto t = [&](int q) { v.targets[v.nt++] = q; };
  auto c = [&](int q) { v.controls[v.nc++] = q; };
  switch (g.code) {
    case G_CX: case G_CZ: case G_CP: case G_CRX: case G_CRY: case G_CRZ: case G_CU:
      c(g.q[0]); t(g.q[1]); break;
    case G_SWAP: case G_ISWAP: case G_RZZ: case G_RXX: case G_RYY: case G_CUSTOM2_FFI: case G_U2_LO:
      t(g.q[0]); t(g.q[1]); break;
    case G_CCX: case G_CCZ:
      c(g.q[0]); c(g.q[1]); t(g.q[2]); break;
    case G_CSWAP:
      c(g.q[0]); t(g.q[1]); t(g.q[2]); break;
    default:
      t(g.q[0]); break;
  }
  return v;
}

bool same_wires(const GateRec& a, const GateRec& b) {
  const View x = view(a), y = view(b);
  if (x.nt != y.nt || x.nc != y.nc) return false;
  for (int i = 0; i < x.nt; ++i)
    if (x.targets[i] != y.targets[i]) return false;
  for (int i = 0; i < x.nc; ++i)
    if (x.controls[i] != y.controls[i]) return false;
  return true;
}

uint64_t wires(const GateRec& g) {
  const View v = view(g);
  uint64_t m = 0;
  for (int i = 0; i < v.nt; ++i) m |= 1ull << v.targets[i];
  for (int i = 0; i < v.nc; ++i) m |= 1ull << v.controls[i];
  return m;
}

bool is_mid(const GateRec& g) { return gate_is_mid(g.code); }
bool one_qubit_plain(const GateRec& g) {  // one target, no controls, a 2x2 matrix
  switch (g.code) {
    case G_H: case G_X: case G_Y: case G_Z: case G_S: case G_T: case G_SX: case G_RX: case G_RY: case G_RZ:
    case G_P: case G_U3: case G_CUSTOM1:
      return true;
    default:
      return false;
  }
}
bool self_inverse_pair(const GateRec& a, const GateRec& b) {
  if (a.code != b.code || !same_wires(a, b)) return false;
  switch (a.code) {
    case G_H: case G_X: case G_Y: case G_Z: case G_CX: case G_CZ: case G_SWAP:
      return true;
    default:
      return false;
  }
}
bool rotation(const GateRec& g) { return g.code == G_RX || g.code == G_RY || g.code == G_RZ; }
bool diagonal(const GateRec& g) {
  return g.code == G_Z || g.code == G_S || g.code == G_T || g.code == G_RZ || g.code == G_P;
}

GateRec mk1(uint8_t code, int q, double p0 = 0.0) {
  GateRec g;
  g.code = code;
  g.nq = uint8_t(gate_arity(code));
  g.q[0] = q;
  g.p[0] = p0;
  return g;
}
GateRec mk2(uint8_t code, int a, int b) {
  GateRec g;
  g.code = code;
  g.nq = 2;
  g.q[0] = a;
  g.q[1] = b;
  return g;
}

std::vector<GateRec> clifford(const std::vector<GateRec>& in, uint64_t* cancellations) {
  std::vector<GateRec> out;
  for (size_t i = 0; i < in.size();) {
    if (i + 1 < in.size() && self_inverse_pair(in[i], in[i + 1])) {
      *cancellations += 2;
      i += 2;
      continue;
    }
    out.push_back(in[i++]);
  }
  return out;
}

std::vector<GateRec> peephole(const std::vector<GateRec>& in, uint64_t* cancellations) {
  std::vector<GateRec> out;
  for (size_t i = 0; i < in.size();) {
    if (i + 2 < in.size()) {
      const GateRec &a = in[i], &b = in[i + 1], &c = in[i + 2];
      if (a.code == G_H && c.code == G_H && (b.code == G_CX || b.code == G_CZ) && a.q[0] == b.q[1] &&
          c.q[0] == b.q[1]) {
        out.push_back(mk2(b.code == G_CX ? G_CZ : G_CX, b.q[0], b.q[1]));
        *cancellations += 2;
        i += 3;
        continue;
      }
      if (a.code == G_CX && b.code == G_X && c.code == G_CX && b.q[0] == a.q[1] && c.q[1] == a.q[1] &&
          c.q[0] == a.q[0]) {
        out.push_back(mk1(G_X, a.q[1]));
        *cancellations += 2;
        i += 3;
        continue;
      }
    }
    if (i + 1 < in.size() && same_wires(in[i], in[i + 1])) {
      const GateRec &a = in[i], &b = in[i + 1];
      if (a.code == G_S && b.code == G_S) {
        out.push_back(mk1(G_Z, a.q[0]));
        *cancellations += 1;
        i += 2;
        continue;
      }
      if (a.code == G_T && b.code == G_T) {
        out.push_back(mk1(G_S, a.q[0]));
        *cancellations += 1;
        i += 2;
        continue;
      }
    }
    out.push_back(in[i++]);
  }
  return out;
}

std::vector<GateRec> merge_rotations(const std::vector<GateRec>& in, uint64_t* fusions) {
  std::vector<GateRec> out;
  for (size_t i = 0; i < in.size();) {
    if (i + 1 < in.size() && rotation(in[i]) && in[i].code == in[i + 1].code && in[i].q[0] == in[i + 1].q[0]) {
      const double a = in[i].p[0] + in[i + 1].p[0];
      if (std::fabs(a) < 1e-10) {
        *fusions += 2;
      } else {
        out.push_back(mk1(in[i].code, in[i].q[0], a));
        *fusions += 1;
      }
      i += 2;
      continue;
    }
    out.push_back(in[i++]);
  }
  return out;
}

bool commute(const GateRec& a, const GateRec& b) {
  if (is_mid(a) || is_mid(b)) return false;
  if (!(wires(a) & wires(b))) return true;
  if (diagonal(a) && diagonal(b)) return true;
  const View va = view(a), vb = view(b);
  auto ctrl_of = [](const View& v, int q) {
    for (int i = 0; i < v.nc; ++i)
      if (v.controls[i] == q) return true;
    return false;
  };
  if (a.code == G_CX && (b.code == G_Z || b.code == G_RZ)) return ctrl_of(va, b.q[0]);
  if (b.code == G_CX && (a.code == G_Z || a.code == G_RZ)) return ctrl_of(vb, a.q[0]);
  if (a.code == G_CX && b.code == G_X) return va.targets[0] == b.q[0];
  if (b.code == G_CX && a.code == G_X) return vb.targets[0] == a.q[0];
  return false;
}

bool cancels_or_merges(const GateRec& a, const GateRec& b) {
  if (!same_wires(a, b)) return false;
  return self_inverse_pair(a, b) || (rotation(a) && a.code == b.code);
}

std::vector<GateRec> commutation(std::vector<GateRec> g, uint64_t* commutations) {
  if (g.size() < 3) return g;
  bool changed = true;
  for (int pass = 0; changed && pass < 5; ++pass) {
    changed = false;
    for (size_t i = 0; i + 1 < g.size(); ++i) {
      if (!commute(g[i], g[i + 1])) continue;
      const bool to_prev = i > 0 && cancels_or_merges(g[i - 1], g[i + 1]);
      const bool to_next = i + 2 < g.size() && cancels_or_merges(g[i], g[i + 2]);
      if (to_prev || to_next) {
        std::swap(g[i], g[i + 1]);
        ++*commutations;
        changed = true;
      }
    }
  }
  return g;
}

// 2x2 matrix of a single-qubit gate, as the engine applies it.
void matrix2(const GateRec& g, cplx* m) {
  const Op o = lower_gate(g);
  if (o.kind == OP_U1) {
    for (int i = 0; i < 4; ++i) m[i] = o.m[i];
  } else if (o.kind == OP_D1) {
    m[0] = o.m[0]; m[1] = 0; m[2] = 0; m[3] = o.m[1];
  } else if (o.kind == OP_PH) {
    m[0] = 1; m[1] = 0; m[2] = 0; m[3] = o.m[0];
  } else {  // OP_X1 (X)
    m[0] = 0; m[1] = 1; m[2] = 1; m[3] = 0;
  }
}

std::vector<GateRec> fuse(const std::vector<GateRec>& in, uint64_t* fusions) {
  std::vector<GateRec> out;
  for (size_t i = 0; i < in.size();) {
    if (!one_qubit_plain(in[i])) {
      out.push_back(in[i++]);
      continue;
    }
    const int q = in[i].q[0];
    size_t j = i;
    while (j < in.size() && one_qubit_plain(in[j]) && in[j].q[0] == q) ++j;
    if (j - i < 2) {
      out.push_back(in[i++]);
      continue;
    }
    cplx u[4];
    matrix2(in[i], u);
    for (size_t k = i + 1; k < j; ++k) {
      cplx m[4], r[4];
      matrix2(in[k], m);
      r[0] = m[0] * u[0] + m[1] * u[2];
      r[1] = m[0] * u[1] + m[1] * u[3];
      r[2] = m[2] * u[0] + m[3] * u[2];
      r[3] = m[2] * u[1] + m[3] * u[3];
      for (int t = 0; t < 4; ++t) u[t] = r[t];
    }
    // identity or global phase (off-diagonals zero, equal diagonal of modulus 1)
    const bool phase_only = std::abs(u[1]) < 1e-10 && std::abs(u[2]) < 1e-10 && std::abs(u[0] - u[3]) < 1e-10 &&
                            std::fabs(std::abs(u[0]) - 1.0) < 1e-10;
    if (phase_only) {
      *fusions += j - i;
    } else {
      GateRec f;
      f.code = G_CUSTOM1;
      f.nq = 1;
      f.q[0] = q;
      for (int t = 0; t < 4; ++t) f.m[t] = u[t];
      out.push_back(f);
      *fusions += j - i - 1;
    }
    i = j;
  }
  return out;
}

}  // namespace
}  // namespace nqpu

using namespace nqpu;

extern "C" NqpuError nqpu_circuit_optimize(NqpuCircuit* circuit, NqpuOptLevel level, uint64_t* stats, uint32_t len) {
  if (!circuit) return NQPU_NULL_POINTER;
  if (level < NQPU_OPT_NONE || level > NQPU_OPT_AGGRESSIVE) return NQPU_INVALID_PARAMETER;
  CircuitImpl* c = reinterpret_cast<CircuitImpl*>(circuit);
  std::lock_guard<std::mutex> lk(c->mu);
  uint64_t fusions = 0, commutations = 0, cancellations = 0;
  const uint64_t original = c->gates.size();
  if (level != NQPU_OPT_NONE && !c->gates.empty()) {
    std::vector<GateRec> g = clifford(c->gates, &cancellations);
    if (level == NQPU_OPT_AGGRESSIVE) g = peephole(g, &cancellations);
    g = merge_rotations(g, &fusions);
    if (level >= NQPU_OPT_MODERATE) g = commutation(g, &commutations);
    g = fuse(g, &fusions);
    g = clifford(g, &cancellations);
    c->gates.swap(g);
    c->version++;
  }
  if (stats) {
    const uint64_t v[6] = {original, c->gates.size(), original - c->gates.size(), fusions, commutations,
                           cancellations};
    for (uint32_t i = 0; i < len && i < 6; ++i) stats[i] = v[i];
  }
  return NQPU_OK;
}

extern "C" NqpuError nqpu_circuit_get_gate(const NqpuCircuit* circuit, uint32_t index, uint32_t* code,
                                           int32_t* qubits, double* params, NqpuComplex* matrix) {
  if (!circuit || !code || !qubits || !params || !matrix) return NQPU_NULL_POINTER;
  const CircuitImpl* c = reinterpret_cast<const CircuitImpl*>(circuit);
  if (index >= c->gates.size()) return NQPU_INVALID_PARAMETER;
  const GateRec& g = c->gates[index];
  *code = g.code;
  for (int i = 0; i < 3; ++i) qubits[i] = g.q[i];
  for (int i = 0; i < 4; ++i) params[i] = g.p[i];
  for (int i = 0; i < 16; ++i) {
    matrix[i].re = g.m[i].real();
    matrix[i].im = g.m[i].imag();
  }
  return NQPU_OK;
}
