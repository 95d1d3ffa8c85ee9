// ORACLE — test infrastructure only.  A CPU restatement of the reference's
// statevector circuit-run path, used by the tests (parity checker), by
// __graft_entry__.smoke() and by bench.py's CPU baseline leg.  Nothing in the
// product library links or calls this code.
//
// Parity pinning: checked against golden vectors produced by the reference's
// own Python statevector (sdk/python/nqpu/core/simulator.py:193-295, generator
// committed at tests/golden/make_golden.py) and against the known-answer tests
// of R/lib.rs:2533-2813 and c_ffi.rs:1646-2660 (restated in tests/).
//
// What it restates (file:line in the reference project):
//   * QuantumState (sdk/rust/src/lib.rs:326-560): |0..0> init, probabilities
//     (:354), fidelity (:388), expectation_z/x/y (:407/:425/:444),
//     expectation_pauli_string (:465), expectation_hamiltonian (:518).
//   * GateOperations (lib.rs:617-1735) per-gate full passes with the same
//     per-amplitude arithmetic: h (:666), x (:712), z (:751), ry (:789),
//     cnot (:835), cz (:880), cphase (:925), s (:1032), t (:1065),
//     rx (:1100), rz (:1146), swap (:1207), toffoli (:1251), u (:1493),
//     u2 (:1536), sx (:1612), phase (:1624), iswap (:1652), ccz (:1688),
//     reset_qubit (:1705); index helpers insert_zero_bit(s) (:575-630).
//   * apply_gate_to_state dispatch (circuits/visualization/ascii_viz.rs:124)
//     with its U3 matrix (:134-150).  Deliberate deviations, applied in both
//     the oracle and the engine: Rzz/Rxx/Ryy use their GateType::matrix
//     (core/gates/gates.rs:440-520) through u2 instead of the dispatcher's
//     no-op; CRx/CRy/CRz use the standard controlled rotations of
//     GateType::matrix; CSWAP and CU (gates.rs:542) are applied.
//   * C FFI custom 2q ordering (infra/bindings/c_ffi.rs:312-395: q1 is the
//     high bit of the sub-index) and sampling (c_ffi.rs:602: first i with
//     r < cumsum_i, else dim-1), xorshift64* RNG (c_ffi.rs:56-66).
//   * GateOpsF32 (core/state_models/quantum_f32.rs:155-700): the same
//     arithmetic in f32 when the state is created with f32 = 1.
// Threading: OpenMP over the same independent index sets the reference splits
// with Rayon (par_iter over dim/2, dim/4 or dim/8 items).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <typename R>
struct Cx {
  R re, im;
};

template <typename R>
inline Cx<R> mul(Cx<R> a, Cx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R>
inline Cx<R> add(Cx<R> a, Cx<R> b) {
  return {a.re + b.re, a.im + b.im};
}

inline uint64_t izb(uint64_t v, int bit) {  // insert_zero_bit, lib.rs:626
  const uint64_t mask = (1ull << bit) - 1;
  return (v & mask) | ((v & ~mask) << 1);
}
inline uint64_t izb2(uint64_t v, int b0, int b1) {  // insert_zero_bits, lib.rs:575 (b0 < b1)
  return izb(izb(v, b0), b1);
}
inline uint64_t izb3(uint64_t v, int b0, int b1, int b2) {  // lib.rs:600
  return izb(izb(izb(v, b0), b1), b2);
}

struct StateBase {
  int n;
  int f32;
  virtual ~StateBase() {}
};

template <typename R>
struct State : StateBase {
  std::vector<Cx<R>> a;
  uint64_t dim() const { return 1ull << n; }
};

// ---- GateOperations restated ------------------------------------------------

// apply_unitary_pair_indexed (lib.rs:634): 2x2 on (i, i|stride)
template <typename R>
void op_u(State<R>& s, int q, const Cx<R> m[4]) {
  const uint64_t half = s.dim() / 2, stride = 1ull << q;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(half); ++k) {
    const uint64_t i = izb(uint64_t(k), q), j = i | stride;
    const Cx<R> x = p[i], y = p[j];
    p[i] = {m[0].re * x.re - m[0].im * x.im + m[1].re * y.re - m[1].im * y.im,
            m[0].re * x.im + m[0].im * x.re + m[1].re * y.im + m[1].im * y.re};
    p[j] = {m[2].re * x.re - m[2].im * x.im + m[3].re * y.re - m[3].im * y.im,
            m[2].re * x.im + m[2].im * x.re + m[3].re * y.im + m[3].im * y.re};
  }
}

template <typename R>
void op_h(State<R>& s, int q) {  // lib.rs:666
  const R inv = R(1) / std::sqrt(R(2));
  const uint64_t half = s.dim() / 2, stride = 1ull << q;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(half); ++k) {
    const uint64_t i = izb(uint64_t(k), q), j = i | stride;
    const Cx<R> x = p[i], y = p[j];
    p[i] = {(x.re + y.re) * inv, (x.im + y.im) * inv};
    p[j] = {(x.re - y.re) * inv, (x.im - y.im) * inv};
  }
}

template <typename R>
void op_x(State<R>& s, int q) {  // lib.rs:712
  const uint64_t half = s.dim() / 2, stride = 1ull << q;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(half); ++k) {
    const uint64_t i = izb(uint64_t(k), q), j = i | stride;
    std::swap(p[i], p[j]);
  }
}

// Y = [[0,-i],[i,0]] as in the C FFI (c_ffi.rs:418) and the Python SDK
// (simulator.py:275).  GateOperations::y (lib.rs:961) applies -Y (the same gate
// up to a global phase of -1); the C FFI form is the one kept here.
template <typename R>
void op_y(State<R>& s, int q) {
  const uint64_t half = s.dim() / 2, stride = 1ull << q;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(half); ++k) {
    const uint64_t i = izb(uint64_t(k), q), j = i | stride;
    const Cx<R> x = p[i], y = p[j];
    p[i] = {y.im, -y.re};
    p[j] = {-x.im, x.re};
  }
}

// diagonal phase on the |1> half (z, s, t, phase: lib.rs:751/1032/1065/1624)
template <typename R>
void op_phase1(State<R>& s, int q, Cx<R> ph) {
  const uint64_t half = s.dim() / 2, stride = 1ull << q;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(half); ++k) {
    const uint64_t j = izb(uint64_t(k), q) | stride;
    p[j] = mul(ph, p[j]);
  }
}

template <typename R>
void op_z(State<R>& s, int q) {  // lib.rs:751 negation
  const uint64_t half = s.dim() / 2, stride = 1ull << q;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(half); ++k) {
    const uint64_t j = izb(uint64_t(k), q) | stride;
    p[j] = {-p[j].re, -p[j].im};
  }
}

template <typename R>
void op_rz(State<R>& s, int q, R theta) {  // lib.rs:1146
  const R c = std::cos(theta / R(2)), sn = std::sin(theta / R(2));
  const Cx<R> p0 = {c, -sn}, p1 = {c, sn};
  const uint64_t half = s.dim() / 2, stride = 1ull << q;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(half); ++k) {
    const uint64_t i = izb(uint64_t(k), q), j = i | stride;
    p[i] = mul(p0, p[i]);
    p[j] = mul(p1, p[j]);
  }
}

template <typename R>
void op_cnot(State<R>& s, int c, int t) {  // lib.rs:835
  const uint64_t quarter = s.dim() / 4;
  const int b0 = c < t ? c : t, b1 = c < t ? t : c;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(quarter); ++k) {
    const uint64_t i = izb2(uint64_t(k), b0, b1) | (1ull << c);
    std::swap(p[i], p[i | (1ull << t)]);
  }
}

// phase on amplitudes with all mask bits set (cz lib.rs:880, cphase :925, ccz :1688)
template <typename R>
void op_phase_mask(State<R>& s, const int* qs, int nq, Cx<R> ph, bool negate) {
  int b[3] = {qs[0], nq > 1 ? qs[1] : 0, nq > 2 ? qs[2] : 0};
  std::sort(b, b + nq);
  uint64_t mask = 0;
  for (int i = 0; i < nq; ++i) mask |= 1ull << qs[i];
  const uint64_t items = s.dim() >> nq;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(items); ++k) {
    uint64_t i = uint64_t(k);
    for (int j = 0; j < nq; ++j) i = izb(i, b[j]);
    i |= mask;
    p[i] = negate ? Cx<R>{-p[i].re, -p[i].im} : mul(ph, p[i]);
  }
}

template <typename R>
void op_swap(State<R>& s, int q1, int q2) {  // lib.rs:1207
  const int lo = q1 < q2 ? q1 : q2, hi = q1 < q2 ? q2 : q1;
  const uint64_t quarter = s.dim() / 4;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(quarter); ++k) {
    const uint64_t base = izb2(uint64_t(k), lo, hi);
    std::swap(p[base | (1ull << lo)], p[base | (1ull << hi)]);
  }
}

template <typename R>
void op_toffoli(State<R>& s, int c1, int c2, int t) {  // lib.rs:1251
  int b[3] = {c1, c2, t};
  std::sort(b, b + 3);
  const uint64_t items = s.dim() / 8;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(items); ++k) {
    const uint64_t i = izb3(uint64_t(k), b[0], b[1], b[2]) | (1ull << c1) | (1ull << c2);
    std::swap(p[i], p[i | (1ull << t)]);
  }
}

template <typename R>
void op_iswap(State<R>& s, int q1, int q2) {  // lib.rs:1652
  const int lo = q1 < q2 ? q1 : q2, hi = q1 < q2 ? q2 : q1;
  const uint64_t quarter = s.dim() / 4;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(quarter); ++k) {
    const uint64_t base = izb2(uint64_t(k), lo, hi);
    const uint64_t i01 = base | (1ull << lo), i10 = base | (1ull << hi);
    const Cx<R> a01 = p[i01], a10 = p[i10];
    p[i01] = {-a10.im, a10.re};
    p[i10] = {-a01.im, a01.re};
  }
}

// GateOperations::u2 (lib.rs:1536): sub-index = (bit(q_hi) << 1) | bit(q_lo)
template <typename R>
void op_u2(State<R>& s, int q_lo, int q_hi, const Cx<R> m[16]) {
  const int b0 = q_lo < q_hi ? q_lo : q_hi, b1 = q_lo < q_hi ? q_hi : q_lo;
  const uint64_t ml = 1ull << q_lo, mh = 1ull << q_hi;
  const uint64_t quarter = s.dim() / 4;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(quarter); ++k) {
    const uint64_t base = izb2(uint64_t(k), b0, b1);
    const uint64_t idx[4] = {base, base | ml, base | mh, base | ml | mh};
    const Cx<R> x[4] = {p[idx[0]], p[idx[1]], p[idx[2]], p[idx[3]]};
    for (int r = 0; r < 4; ++r) {
      Cx<R> acc = mul(m[r * 4 + 0], x[0]);
      acc = add(acc, mul(m[r * 4 + 1], x[1]));
      acc = add(acc, mul(m[r * 4 + 2], x[2]));
      acc = add(acc, mul(m[r * 4 + 3], x[3]));
      p[idx[r]] = acc;
    }
  }
}

// controlled 2x2 (standard CRx/CRy/CRz/CU of GateType::matrix, gates.rs)
template <typename R>
void op_cu(State<R>& s, int c, int t, const Cx<R> m[4]) {
  const int b0 = c < t ? c : t, b1 = c < t ? t : c;
  const uint64_t quarter = s.dim() / 4;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(quarter); ++k) {
    const uint64_t i = izb2(uint64_t(k), b0, b1) | (1ull << c), j = i | (1ull << t);
    const Cx<R> x = p[i], y = p[j];
    p[i] = add(mul(m[0], x), mul(m[1], y));
    p[j] = add(mul(m[2], x), mul(m[3], y));
  }
}

template <typename R>
void op_cswap(State<R>& s, int c, int q1, int q2) {
  int b[3] = {c, q1, q2};
  std::sort(b, b + 3);
  const uint64_t items = s.dim() / 8;
  Cx<R>* p = s.a.data();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < int64_t(items); ++k) {
    const uint64_t base = izb3(uint64_t(k), b[0], b[1], b[2]) | (1ull << c);
    std::swap(p[base | (1ull << q1)], p[base | (1ull << q2)]);
  }
}

template <typename R>
void op_reset_qubit(State<R>& s, int q) {  // lib.rs:1705
  const uint64_t mask = 1ull << q;
  Cx<R>* p = s.a.data();
  const int64_t dim = int64_t(s.dim());
  for (int64_t i = 0; i < dim; ++i)
    if (uint64_t(i) & mask) p[i] = {R(0), R(0)};
  R norm = 0;
  for (int64_t i = 0; i < dim; ++i) norm += p[i].re * p[i].re + p[i].im * p[i].im;
  norm = std::sqrt(norm);
  if (norm > 0) {
    const R inv = R(1) / norm;
    for (int64_t i = 0; i < dim; ++i) { p[i].re *= inv; p[i].im *= inv; }
  }
}

// ---- gate dispatch (apply_gate_to_state, ascii_viz.rs:124) -----------------
enum Code {
  H, X, Y, Z, S, T, SX, RX, RY, RZ, P, U3, CX, CZ, SWAP, ISWAP, CP, CRX, CRY, CRZ, RZZ, RXX, RYY,
  CCX, CCZ, CSWAP, CUSTOM1, CUSTOM2, U2LO, CU, MEASURE, RESET
};

}  // namespace
extern "C" double oracle_next_random();  // xorshift64* draw (c_ffi.rs:56-66)
namespace {
std::vector<uint32_t> g_outcomes;      // outcomes of MEASURE gates, in order

// Mid-circuit measurement (QuantumSimulator::measure_qubit, lib.rs:1835, with
// the C FFI's probability rule, c_ffi.rs:537-560): P(0) summed over the |0>
// half, outcome 0 iff r < P(0), the other half zeroed and the kept half scaled
// by 1/sqrt(P(outcome)).
template <typename R>
void op_measure(State<R>& s, int q) {
  const uint64_t mask = 1ull << q;
  double p0 = 0.0;
  for (uint64_t i = 0; i < s.dim(); ++i)
    if (!(i & mask)) p0 += double(s.a[i].re) * s.a[i].re + double(s.a[i].im) * s.a[i].im;
  const double r = oracle_next_random();
  const uint32_t out = r < p0 ? 0u : 1u;
  const double po = out == 0 ? p0 : 1.0 - p0;
  const R f = R(1.0 / std::sqrt(po));
  for (uint64_t i = 0; i < s.dim(); ++i) {
    if (((i & mask) != 0) != (out == 1)) s.a[i] = {R(0), R(0)};
    else { s.a[i].re *= f; s.a[i].im *= f; }
  }
  g_outcomes.push_back(out);
}

template <typename R>
void apply_flat(State<R>& s, const double* g) {
  const int code = int(g[0]);
  const int a = int(g[1]), b = int(g[2]), c = int(g[3]);
  const double th = g[4], ph = g[5], la = g[6], ga = g[7];
  auto M = [&](int i) { return Cx<R>{R(g[8 + 2 * i]), R(g[9 + 2 * i])}; };
  switch (code) {
    case MEASURE: op_measure(s, a); break;
    case RESET: {  // OpenQASM reset: measure (not recorded), flip back to |0> on 1
      const size_t k = g_outcomes.size();
      op_measure(s, a);
      const uint32_t out = g_outcomes.back();
      g_outcomes.resize(k);
      if (out == 1) op_x(s, a);
      break;
    }
    case H: op_h(s, a); break;
    case X: op_x(s, a); break;
    case Y: op_y(s, a); break;
    case Z: op_z(s, a); break;
    case S: op_phase1(s, a, Cx<R>{R(0), R(1)}); break;
    case T: {
      const double q = 0.78539816339744830962;  // FRAC_PI_4
      op_phase1(s, a, Cx<R>{R(std::cos(q)), R(std::sin(q))});
      break;
    }
    case SX: {
      const Cx<R> m[4] = {{R(0.5), R(0.5)}, {R(0.5), R(-0.5)}, {R(0.5), R(-0.5)}, {R(0.5), R(0.5)}};
      op_u(s, a, m);
      break;
    }
    case RX: {
      const R cs = R(std::cos(th / 2.0)), sn = R(std::sin(th / 2.0));
      const Cx<R> m[4] = {{cs, 0}, {0, -sn}, {0, -sn}, {cs, 0}};
      op_u(s, a, m);
      break;
    }
    case RY: {
      const R cs = R(std::cos(th / 2.0)), sn = R(std::sin(th / 2.0));
      const Cx<R> m[4] = {{cs, 0}, {-sn, 0}, {sn, 0}, {cs, 0}};
      op_u(s, a, m);
      break;
    }
    case RZ: op_rz(s, a, R(th)); break;
    case P: op_phase1(s, a, Cx<R>{R(std::cos(th)), R(std::sin(th))}); break;
    case U3: {  // ascii_viz.rs:134-150
      const double cs = std::cos(th / 2.0), sn = std::sin(th / 2.0);
      const Cx<R> m[4] = {{R(cs), R(0)},
                          {R(-sn * std::cos(la)), R(-sn * std::sin(la))},
                          {R(sn * std::cos(ph)), R(sn * std::sin(ph))},
                          {R(cs * std::cos(ph + la)), R(cs * std::sin(ph + la))}};
      op_u(s, a, m);
      break;
    }
    case CX: op_cnot(s, a, b); break;
    case CZ: { int qs[2] = {a, b}; op_phase_mask(s, qs, 2, Cx<R>{}, true); break; }
    case SWAP: op_swap(s, a, b); break;
    case ISWAP: op_iswap(s, a, b); break;
    case CP: { int qs[2] = {a, b}; op_phase_mask(s, qs, 2, Cx<R>{R(std::cos(th)), R(std::sin(th))}, false); break; }
    case CRX: {
      const R cs = R(std::cos(th / 2.0)), sn = R(std::sin(th / 2.0));
      const Cx<R> m[4] = {{cs, 0}, {0, -sn}, {0, -sn}, {cs, 0}};
      op_cu(s, a, b, m);
      break;
    }
    case CRY: {
      const R cs = R(std::cos(th / 2.0)), sn = R(std::sin(th / 2.0));
      const Cx<R> m[4] = {{cs, 0}, {-sn, 0}, {sn, 0}, {cs, 0}};
      op_cu(s, a, b, m);
      break;
    }
    case CRZ: {
      const Cx<R> m[4] = {{R(std::cos(-th / 2)), R(std::sin(-th / 2))}, {0, 0}, {0, 0},
                          {R(std::cos(th / 2)), R(std::sin(th / 2))}};
      op_cu(s, a, b, m);
      break;
    }
    case RZZ: {  // gates.rs:486 through u2
      const R cs = R(std::cos(th / 2.0)), sn = R(std::sin(th / 2.0));
      Cx<R> m[16] = {};
      m[0] = {cs, -sn}; m[5] = {cs, sn}; m[10] = {cs, sn}; m[15] = {cs, -sn};
      op_u2(s, a, b, m);
      break;
    }
    case RXX: {
      const R cs = R(std::cos(th / 2.0)), sn = R(std::sin(th / 2.0));
      Cx<R> m[16] = {};
      m[0] = m[5] = m[10] = m[15] = {cs, 0};
      m[3] = m[6] = m[9] = m[12] = {0, -sn};
      op_u2(s, a, b, m);
      break;
    }
    case RYY: {
      const R cs = R(std::cos(th / 2.0)), sn = R(std::sin(th / 2.0));
      Cx<R> m[16] = {};
      m[0] = m[5] = m[10] = m[15] = {cs, 0};
      m[3] = m[12] = {0, sn};
      m[6] = m[9] = {0, -sn};
      op_u2(s, a, b, m);
      break;
    }
    case CCX: op_toffoli(s, a, b, c); break;
    case CCZ: { int qs[3] = {a, b, c}; op_phase_mask(s, qs, 3, Cx<R>{}, true); break; }
    case CSWAP: op_cswap(s, a, b, c); break;
    case CUSTOM1: { const Cx<R> m[4] = {M(0), M(1), M(2), M(3)}; op_u(s, a, m); break; }
    case CUSTOM2: {
      // c_ffi apply_2q: basis |q1 q2>, q1 high -> u2 with q_lo = q2, q_hi = q1
      Cx<R> m[16];
      for (int i = 0; i < 16; ++i) m[i] = M(i);
      op_u2(s, b, a, m);
      break;
    }
    case U2LO: {
      Cx<R> m[16];
      for (int i = 0; i < 16; ++i) m[i] = M(i);
      op_u2(s, a, b, m);
      break;
    }
    case CU: {  // gates.rs:542
      const double cs = std::cos(th / 2.0), sn = std::sin(th / 2.0);
      const Cx<R> m[4] = {{R(std::cos(ga) * cs), R(std::sin(ga) * cs)},
                          {R(-std::cos(ga + la) * sn), R(-std::sin(ga + la) * sn)},
                          {R(std::cos(ga + ph) * sn), R(std::sin(ga + ph) * sn)},
                          {R(std::cos(ga + ph + la) * cs), R(std::sin(ga + ph + la) * cs)}};
      op_cu(s, a, b, m);
      break;
    }
    default: break;
  }
}

thread_local uint64_t rng_state = 0x853c49e6748fea9bull;

template <typename F>
auto with_state(void* h, F&& f) {
  StateBase* b = static_cast<StateBase*>(h);
  if (b->f32) return f(*static_cast<State<float>*>(b));
  return f(*static_cast<State<double>*>(b));
}

}  // namespace

extern "C" {

void oracle_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}

int oracle_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void* oracle_state_new(int n, int f32) {
  StateBase* s;
  if (f32) {
    auto* t = new State<float>();
    t->a.assign(1ull << n, Cx<float>{0, 0});
    t->a[0] = {1, 0};
    s = t;
  } else {
    auto* t = new State<double>();
    t->a.assign(1ull << n, Cx<double>{0, 0});
    t->a[0] = {1, 0};
    s = t;
  }
  s->n = n;
  s->f32 = f32;
  return s;
}

void oracle_state_free(void* h) { delete static_cast<StateBase*>(h); }

void oracle_state_set_basis(void* h, uint64_t idx) {
  with_state(h, [&](auto& s) {
    using R = decltype(s.a[0].re);
    std::fill(s.a.begin(), s.a.end(), Cx<R>{0, 0});
    s.a[idx] = {R(1), R(0)};
    return 0;
  });
}

// out: 2*dim doubles (re, im)
void oracle_state_get(void* h, double* out) {
  with_state(h, [&](auto& s) {
    for (uint64_t i = 0; i < s.dim(); ++i) { out[2 * i] = s.a[i].re; out[2 * i + 1] = s.a[i].im; }
    return 0;
  });
}

void oracle_state_set(void* h, const double* in) {
  with_state(h, [&](auto& s) {
    using R = decltype(s.a[0].re);
    for (uint64_t i = 0; i < s.dim(); ++i) s.a[i] = {R(in[2 * i]), R(in[2 * i + 1])};
    return 0;
  });
}

// flat: ngates x 40 doubles (code, q0, q1, q2, p0..p3, 16 complex matrix)
void oracle_apply_flat(void* h, const double* flat, int ngates) {
  with_state(h, [&](auto& s) {
    for (int i = 0; i < ngates; ++i) apply_flat(s, flat + size_t(i) * 40);
    return 0;
  });
}

void oracle_reset_qubit(void* h, int q) {
  with_state(h, [&](auto& s) { op_reset_qubit(s, q); return 0; });
}

// QuantumState::expectation_z (lib.rs:407) for every qubit: serial loop per qubit.
void oracle_expectation_z_all(void* h, double* out) {
  with_state(h, [&](auto& s) {
    for (int q = 0; q < s.n; ++q) {
      const uint64_t stride = 1ull << q;
      double e = 0.0;
      for (uint64_t i = 0; i < s.dim(); ++i) {
        const double pr = double(s.a[i].re) * s.a[i].re + double(s.a[i].im) * s.a[i].im;
        if (i & stride) e -= pr; else e += pr;
      }
      out[q] = e;
    }
    return 0;
  });
}

double oracle_expectation_x(void* h, int q) {  // lib.rs:425
  return with_state(h, [&](auto& s) {
    const uint64_t stride = 1ull << q;
    double e = 0.0;
    for (uint64_t i = 0; i < s.dim(); ++i)
      if (!(i & stride)) {
        const auto ai = s.a[i], aj = s.a[i | stride];
        e += 2.0 * (double(ai.re) * aj.re + double(ai.im) * aj.im);
      }
    return e;
  });
}

double oracle_expectation_y(void* h, int q) {  // lib.rs:444
  return with_state(h, [&](auto& s) {
    const uint64_t stride = 1ull << q;
    double e = 0.0;
    for (uint64_t i = 0; i < s.dim(); ++i)
      if (!(i & stride)) {
        const auto ai = s.a[i], aj = s.a[i | stride];
        e += 2.0 * (double(aj.re) * ai.im - double(aj.im) * ai.re);
      }
    return e;
  });
}

// lib.rs:465; `ops` has `len` chars, char q acts on qubit q
double oracle_pauli_string(void* h, const char* ops, int len) {
  return with_state(h, [&](auto& s) {
    double result = 0.0;
    for (uint64_t i = 0; i < s.dim(); ++i) {
      uint64_t j = i;
      double cr = 1.0, ci = 0.0;
      for (int q = 0; q < len; ++q) {
        const int bit = int((i >> q) & 1);
        switch (ops[q]) {
          case 'X': j ^= 1ull << q; break;
          case 'Y': {
            j ^= 1ull << q;
            double nr, ni;
            if (bit == 0) { nr = -ci; ni = cr; } else { nr = ci; ni = -cr; }
            cr = nr; ci = ni;
            break;
          }
          case 'Z': if (bit) { cr = -cr; ci = -ci; } break;
          default: break;
        }
      }
      const auto ai = s.a[i], aj = s.a[j];
      const double pr = cr * aj.re - ci * aj.im;
      const double pi = cr * aj.im + ci * aj.re;
      result += ai.re * pr + ai.im * pi;
    }
    return result;
  });
}

double oracle_norm(void* h) {
  return with_state(h, [&](auto& s) {
    double t = 0.0;
    for (uint64_t i = 0; i < s.dim(); ++i) t += double(s.a[i].re) * s.a[i].re + double(s.a[i].im) * s.a[i].im;
    return t;
  });
}

// lib.rs:388 |<a|b>|^2 (either precision)
double oracle_fidelity(void* ha, void* hb) {
  StateBase* A = static_cast<StateBase*>(ha);
  StateBase* B = static_cast<StateBase*>(hb);
  if (A->n != B->n) return 0.0;
  const uint64_t dim = 1ull << A->n;
  auto get = [](StateBase* s, uint64_t i, double* r, double* m) {
    if (s->f32) { auto& t = *static_cast<State<float>*>(s); *r = t.a[i].re; *m = t.a[i].im; }
    else { auto& t = *static_cast<State<double>*>(s); *r = t.a[i].re; *m = t.a[i].im; }
  };
  double re = 0.0, im = 0.0;
  for (uint64_t i = 0; i < dim; ++i) {
    double ar, ai, br, bi;
    get(A, i, &ar, &ai);
    get(B, i, &br, &bi);
    re += ar * br + ai * bi;
    im += ar * bi - ai * br;
  }
  return re * re + im * im;
}

void oracle_probabilities(void* h, double* out) {  // lib.rs:354
  with_state(h, [&](auto& s) {
    for (uint64_t i = 0; i < s.dim(); ++i) out[i] = double(s.a[i].re) * s.a[i].re + double(s.a[i].im) * s.a[i].im;
    return 0;
  });
}

// c_ffi.rs:602 sample with given uniforms: first i with r < cumsum_i, else dim-1.
void oracle_sample_uniforms(void* h, const double* u, int shots, uint64_t* out) {
  with_state(h, [&](auto& s) {
    std::vector<double> cdf(s.dim());
    double c = 0.0;
    for (uint64_t i = 0; i < s.dim(); ++i) {
      c += double(s.a[i].re) * s.a[i].re + double(s.a[i].im) * s.a[i].im;
      cdf[i] = c;
    }
    for (int k = 0; k < shots; ++k) {
      const double r = u[k];
      auto it = std::upper_bound(cdf.begin(), cdf.end(), r);  // first cdf > r
      out[k] = it == cdf.end() ? s.dim() - 1 : uint64_t(it - cdf.begin());
    }
    return 0;
  });
}

// outcomes of the MEASURE gates applied since the last call (up to max)
int oracle_take_outcomes(uint32_t* out, int max) {
  const int k = int(std::min<size_t>(g_outcomes.size(), size_t(max)));
  for (int i = 0; i < k; ++i) out[i] = g_outcomes[size_t(i)];
  g_outcomes.clear();
  return k;
}

// xorshift64* of c_ffi.rs:56-66 and nqpu_set_seed (c_ffi.rs:1444)
void oracle_set_seed(uint64_t seed) { rng_state = seed == 0 ? 0x853c49e6748fea9bull : seed; }
double oracle_next_random() {
  uint64_t s = rng_state;
  s ^= s >> 12;
  s ^= s << 25;
  s ^= s >> 27;
  rng_state = s;
  const uint64_t v = s * 0x2545F4914F6CDD1Dull;
  return double(v >> 11) / double(1ull << 53);
}

}  // extern "C"
