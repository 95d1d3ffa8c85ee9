// Gate lowering and the tiled-pass planner.
//
// Lowering follows the reference's matrices:
//   * 1q gates: GateOperations (R/lib.rs:666-1140) / the C FFI gate_* bodies
//     (c_ffi.rs:400-470); U3 from apply_gate_to_state (ascii_viz.rs:134-150);
//     SX from GateOperations::sx (R/lib.rs:1612).
//   * 2q/3q gates: GateType::matrix (gates.rs:70-600).  Rzz/Rxx/Ryy are applied
//     with their gates.rs matrices (the reference dispatcher drops them,
//     ascii_viz.rs:166); CRx/CRy/CRz use the standard controlled rotations of
//     GateType::matrix, not GateOperations::crx/cry/crz.
//
// Planner: greedy grouping of ops into HBM passes (tile-qubit sets) and of a
// pass's ops into register stages.  An op may move ahead of an earlier op that
// stays behind only when the two share no qubit (so they commute).
#include "planner.h"
#include <algorithm>
#include <cmath>
#include <iterator>
#include <cstring>

namespace nqpu {

int gate_arity(uint8_t code) {
  switch (code) {
    case G_CX: case G_CZ: case G_SWAP: case G_ISWAP: case G_CP: case G_CRX: case G_CRY:
    case G_CRZ: case G_RZZ: case G_RXX: case G_RYY: case G_CUSTOM2_FFI: case G_U2_LO: case G_CU:
      return 2;
    case G_CCX: case G_CCZ: case G_CSWAP:
      return 3;
    default:
      return 1;
  }
}

bool gate_has_params(uint8_t code) {
  switch (code) {
    case G_RX: case G_RY: case G_RZ: case G_P: case G_U3: case G_CP: case G_CRX: case G_CRY:
    case G_CRZ: case G_RZZ: case G_RXX: case G_RYY: case G_CU:
      return true;
    default:
      return false;
  }
}

static cplx expi(double a) { return cplx(std::cos(a), std::sin(a)); }

static void set1(Op& o, cplx a, cplx b, cplx c, cplx d) {
  o.m[0] = a; o.m[1] = b; o.m[2] = c; o.m[3] = d;
}

static void rx_m(Op& o, double th) {
  const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
  set1(o, cplx(c, 0), cplx(0, -s), cplx(0, -s), cplx(c, 0));
}
static void ry_m(Op& o, double th) {
  const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
  set1(o, cplx(c, 0), cplx(-s, 0), cplx(s, 0), cplx(c, 0));
}

Op lower_gate(const GateRec& g) {
  Op o;
  const int a = g.q[0], b = g.q[1], c3 = g.q[2];
  const double th = g.p[0];
  switch (g.code) {
    case G_H: {
      const double s = 0.70710678118654752440;  // FRAC_1_SQRT_2 (c_ffi.rs:402)
      o.kind = OP_U1; o.t0 = a;
      set1(o, cplx(s, 0), cplx(s, 0), cplx(s, 0), cplx(-s, 0));
      break;
    }
    case G_X: o.kind = OP_X1; o.t0 = a; break;
    case G_Y:
      o.kind = OP_U1; o.t0 = a;
      set1(o, cplx(0, 0), cplx(0, -1), cplx(0, 1), cplx(0, 0));
      break;
    case G_Z: o.kind = OP_PH; o.t0 = a; o.m[0] = cplx(-1, 0); break;
    case G_S: o.kind = OP_PH; o.t0 = a; o.m[0] = cplx(0, 1); break;
    case G_T: {
      const double q = 0.78539816339744830962;  // FRAC_PI_4 (c_ffi.rs:434)
      o.kind = OP_PH; o.t0 = a; o.m[0] = cplx(std::cos(q), std::sin(q));
      break;
    }
    case G_SX:
      o.kind = OP_U1; o.t0 = a;
      set1(o, cplx(0.5, 0.5), cplx(0.5, -0.5), cplx(0.5, -0.5), cplx(0.5, 0.5));
      break;
    case G_RX: o.kind = OP_U1; o.t0 = a; rx_m(o, th); break;
    case G_RY: o.kind = OP_U1; o.t0 = a; ry_m(o, th); break;
    case G_RZ: {
      const double h = th / 2.0;
      o.kind = OP_D1; o.t0 = a;
      o.m[0] = cplx(std::cos(h), -std::sin(h));
      o.m[1] = cplx(std::cos(h), std::sin(h));
      break;
    }
    case G_P: o.kind = OP_PH; o.t0 = a; o.m[0] = cplx(std::cos(th), std::sin(th)); break;
    case G_U3: {
      const double phi = g.p[1], lam = g.p[2];
      const double cs = std::cos(th / 2.0), sn = std::sin(th / 2.0);
      o.kind = OP_U1; o.t0 = a;
      set1(o, cplx(cs, 0.0), cplx(-sn * std::cos(lam), -sn * std::sin(lam)),
           cplx(sn * std::cos(phi), sn * std::sin(phi)),
           cplx(cs * std::cos(phi + lam), cs * std::sin(phi + lam)));
      break;
    }
    case G_CX: o.kind = OP_X1; o.t0 = b; o.nctrl = 1; o.ctrl[0] = a; break;
    case G_CZ: o.kind = OP_PH; o.t0 = b; o.nctrl = 1; o.ctrl[0] = a; o.m[0] = cplx(-1, 0); break;
    case G_SWAP: o.kind = OP_SW; o.t0 = a; o.t1 = b; break;
    case G_ISWAP:
      o.kind = OP_U2; o.t0 = a; o.t1 = b;
      for (auto& v : o.m) v = 0;
      o.m[0] = 1; o.m[15] = 1;
      o.m[1 * 4 + 2] = cplx(0, 1);  // |10> (sub 2) -> i|01> (sub 1)
      o.m[2 * 4 + 1] = cplx(0, 1);  // |01> (sub 1) -> i|10> (sub 2)
      break;
    case G_CP: o.kind = OP_PH; o.t0 = b; o.nctrl = 1; o.ctrl[0] = a; o.m[0] = expi(th); break;
    case G_CRX: o.kind = OP_U1; o.t0 = b; o.nctrl = 1; o.ctrl[0] = a; rx_m(o, th); break;
    case G_CRY: o.kind = OP_U1; o.t0 = b; o.nctrl = 1; o.ctrl[0] = a; ry_m(o, th); break;
    case G_CRZ:
      o.kind = OP_D1; o.t0 = b; o.nctrl = 1; o.ctrl[0] = a;
      o.m[0] = expi(-th / 2.0); o.m[1] = expi(th / 2.0);
      break;
    case G_RZZ: {
      // gates.rs:486 diag(e^{-i th/2}, e^{i th/2}, e^{i th/2}, e^{-i th/2})
      const double cs = std::cos(th / 2.0), sn = std::sin(th / 2.0);
      o.kind = OP_D2; o.t0 = a; o.t1 = b;
      o.m[0] = cplx(cs, -sn); o.m[1] = cplx(cs, sn); o.m[2] = cplx(cs, sn); o.m[3] = cplx(cs, -sn);
      break;
    }
    case G_RXX: {
      const double cs = std::cos(th / 2.0), sn = std::sin(th / 2.0);
      o.kind = OP_U2; o.t0 = a; o.t1 = b;
      for (auto& v : o.m) v = 0;
      o.m[0] = o.m[5] = o.m[10] = o.m[15] = cplx(cs, 0);
      o.m[3] = o.m[6] = o.m[9] = o.m[12] = cplx(0, -sn);
      break;
    }
    case G_RYY: {
      const double cs = std::cos(th / 2.0), sn = std::sin(th / 2.0);
      o.kind = OP_U2; o.t0 = a; o.t1 = b;
      for (auto& v : o.m) v = 0;
      o.m[0] = o.m[5] = o.m[10] = o.m[15] = cplx(cs, 0);
      o.m[3] = o.m[12] = cplx(0, sn);
      o.m[6] = o.m[9] = cplx(0, -sn);
      break;
    }
    case G_CCX: o.kind = OP_X1; o.t0 = c3; o.nctrl = 2; o.ctrl[0] = a; o.ctrl[1] = b; break;
    case G_CCZ:
      o.kind = OP_PH; o.t0 = c3; o.nctrl = 2; o.ctrl[0] = a; o.ctrl[1] = b; o.m[0] = cplx(-1, 0);
      break;
    case G_CSWAP: o.kind = OP_SW; o.t0 = b; o.t1 = c3; o.nctrl = 1; o.ctrl[0] = a; break;
    case G_CUSTOM1: o.kind = OP_U1; o.t0 = a; for (int i = 0; i < 4; ++i) o.m[i] = g.m[i]; break;
    case G_CUSTOM2_FFI:
      // c_ffi.rs:312-395: basis |q1 q2>, q1 is the high sub-index bit.
      o.kind = OP_U2; o.t0 = b; o.t1 = a;
      for (int i = 0; i < 16; ++i) o.m[i] = g.m[i];
      break;
    case G_U2_LO:
      // R/lib.rs:1536: qubit_lo is bit 0 of the sub-index.
      o.kind = OP_U2; o.t0 = a; o.t1 = b;
      for (int i = 0; i < 16; ++i) o.m[i] = g.m[i];
      break;
    case G_CU: {
      // gates.rs:542: |0><0| x I + e^{i gamma} |1><1| x U3(theta, phi, lambda)
      const double phi = g.p[1], lam = g.p[2], gam = g.p[3];
      const double cs = std::cos(th / 2.0), sn = std::sin(th / 2.0);
      o.kind = OP_U1; o.t0 = b; o.nctrl = 1; o.ctrl[0] = a;
      set1(o, cplx(std::cos(gam) * cs, std::sin(gam) * cs),
           cplx(-std::cos(gam + lam) * sn, -std::sin(gam + lam) * sn),
           cplx(std::cos(gam + phi) * sn, std::sin(gam + phi) * sn),
           cplx(std::cos(gam + phi + lam) * cs, std::sin(gam + phi + lam) * cs));
      break;
    }
    default:
      break;
  }
  return o;
}

std::vector<Op> lower_circuit(const std::vector<GateRec>& gates) {
  std::vector<Op> ops;
  ops.reserve(gates.size());
  for (const auto& g : gates) ops.push_back(lower_gate(g));
  return ops;
}

uint32_t circuit_depth(const std::vector<GateRec>& gates, uint32_t n) {
  if (gates.empty()) return 0;
  std::vector<uint32_t> qd(n, 0);
  uint32_t mx = 0;
  for (const auto& g : gates) {
    const int ar = gate_arity(g.code);
    uint32_t layer = 0;
    for (int i = 0; i < ar; ++i) layer = std::max(layer, qd[g.q[i]]);
    for (int i = 0; i < ar; ++i) qd[g.q[i]] = layer + 1;
    mx = std::max(mx, layer + 1);
  }
  return mx;
}

// ---------------------------------------------------------------------------
// Tiled pass planner
// ---------------------------------------------------------------------------

int tile_min_qubits(DType dt) { return dt == DType::C64 ? 5 : 4; }

static int popc(uint64_t x) { return __builtin_popcountll(x); }

static uint64_t dense_targets(const Op& o) {
  uint64_t m = 0;
  if (o.n_targets() >= 1) m |= 1ull << o.t0;
  if (o.n_targets() >= 2) m |= 1ull << o.t1;
  return m;
}

// Qubits whose bit value the op reads without being a register target
// (controls, diagonal qubits, the PH target).
static uint64_t value_qubits(const Op& o) {
  uint64_t m = o.ctrl_mask();
  if (o.kind == OP_D1 || o.kind == OP_PH) m |= 1ull << o.t0;
  if (o.kind == OP_D2) m |= (1ull << o.t0) | (1ull << o.t1);
  return m;
}

template <typename Real>
static TileOp<Real> encode_op(const Op& o, const int* tile_pos, const int* reg_of_tile,
                              const int* ext_of_qubit, int k) {
  TileOp<Real> t;
  std::memset(&t, 0, sizeof(t));
  t.kind = o.kind;
  t.dreg0 = t.dreg1 = 0xFF;
  auto vmask = [&](int q, uint8_t* creg, uint32_t* cnr) {
    const int tb = tile_pos[q];
    if (tb >= 0) {
      if (reg_of_tile[tb] >= 0) *creg |= uint8_t(1u << reg_of_tile[tb]);
      else *cnr |= 1u << tb;
    } else {
      *cnr |= 1u << (k + ext_of_qubit[q]);
    }
  };
  uint8_t creg = 0;
  uint32_t cnr = 0;
  for (int i = 0; i < o.nctrl; ++i) vmask(o.ctrl[i], &creg, &cnr);
  if (o.kind == OP_PH) vmask(o.t0, &creg, &cnr);
  t.creg = creg;
  t.cnr = cnr;
  if (o.kind == OP_U1 || o.kind == OP_X1 || o.kind == OP_U2 || o.kind == OP_SW) {
    t.rb0 = uint8_t(reg_of_tile[tile_pos[o.t0]]);
    if (o.kind == OP_U2 || o.kind == OP_SW) t.rb1 = uint8_t(reg_of_tile[tile_pos[o.t1]]);
  }
  auto diag = [&](int q, uint8_t* dreg, uint32_t* dv) {
    const int tb = tile_pos[q];
    if (tb >= 0 && reg_of_tile[tb] >= 0) {
      *dreg = uint8_t(reg_of_tile[tb]);
    } else {
      *dreg = 0xFF;
      *dv = tb >= 0 ? (1u << tb) : (1u << (k + ext_of_qubit[q]));
    }
  };
  if (o.kind == OP_D1) diag(o.t0, &t.dreg0, &t.dv0);
  if (o.kind == OP_D2) { diag(o.t0, &t.dreg0, &t.dv0); diag(o.t1, &t.dreg1, &t.dv1); }
  for (int i = 0; i < 16; ++i) {
    t.m[2 * i] = Real(o.m[i].real());
    t.m[2 * i + 1] = Real(o.m[i].imag());
  }
  // flat dispatch code: 1 + b for a dense 1q gate on register bit b without
  // register controls, 8 + 8 b + v for X on register bit b with at most one
  // register control (v = 0: none, else its register bit + 1)
  if (o.kind == OP_U1 && t.creg == 0) t.fast = uint8_t(1 + t.rb0);
  if (o.kind == OP_X1 && (t.creg & (t.creg - 1)) == 0) {
    int v = 0;
    if (t.creg) {
      v = 1;
      while (!((t.creg >> (v - 1)) & 1u)) ++v;
    }
    t.fast = uint8_t(8 + 8 * t.rb0 + v);
  }
  // Diagonal shapes (read by the batch executor, whose HEA circuits are two
  // thirds diagonal ops; d = register bit, nrb for a thread-level bit):
  //   48 + d           diag(d0, d1) on bit d, no controls
  //   128 + creg       phase on register mask creg (controls outside the registers: tc)
  //   160 + 8 d0 + d1  diagonal on bits (d0, d1), no controls
  const int nrb = sizeof(Real) == 4 ? 5 : 4;
  auto dbit = [&](uint8_t d) { return d == 0xFF ? nrb : int(d); };
  if (o.kind == OP_D1 && t.creg == 0 && t.cnr == 0) t.fast2 = uint8_t(48 + dbit(t.dreg0));
  if (o.kind == OP_PH) t.fast2 = uint8_t(128 + t.creg);
  if (o.kind == OP_D2 && t.creg == 0 && t.cnr == 0) t.fast2 = uint8_t(160 + 8 * dbit(t.dreg0) + dbit(t.dreg1));
  return t;
}

bool build_tile_plan(const std::vector<Op>& ops, int n, DType dt, int kmax, TilePlan* out,
                     std::string* err) {
  const int vb = dt == DType::C64 ? 1 : 0;
  out->dt = dt;
  out->n = n;
  out->passes.clear();
  out->stages.clear();
  out->ops_f.clear();
  out->ops_d.clear();
  if (n < tile_min_qubits(dt)) {
    if (err) *err = "state too small for the tiled kernel";
    return false;
  }
  const int k = std::min(kmax, n);
  const int c = std::min(k, dt == DType::C64 ? 5 : 4);
  const uint64_t all = (n >= 64) ? ~0ull : ((1ull << n) - 1);
  const uint64_t lowc = (1ull << c) - 1;

  std::vector<int> remaining(ops.size());
  for (size_t i = 0; i < ops.size(); ++i) remaining[i] = int(i);

  while (!remaining.empty()) {
    uint64_t Q = (n <= kmax) ? all : lowc;
    uint64_t blocked = 0, used_val = 0;
    std::vector<int> taken, rest;
    for (int idx : remaining) {
      const Op& o = ops[idx];
      const uint64_t qm = o.qubit_mask();
      if (qm & blocked) { blocked |= qm; rest.push_back(idx); continue; }
      const uint64_t need = dense_targets(o) & ~Q;
      const uint64_t nQ = Q | need;
      const uint64_t nval = used_val | value_qubits(o);
      const bool fits = popc(nQ) <= k && popc(nval & ~nQ) <= 32 - k;
      if (fits) {
        Q = nQ;
        used_val = nval;
        taken.push_back(idx);
      } else {
        blocked |= qm;
        rest.push_back(idx);
      }
    }
    // Fill Q up to k qubits: prefer qubits read as values by taken ops (fewer
    // ext bits), then the lowest unused qubits.
    for (int q = 0; q < n && popc(Q) < k; ++q)
      if (((used_val >> q) & 1) && !((Q >> q) & 1)) Q |= 1ull << q;
    for (int q = 0; q < n && popc(Q) < k; ++q) Q |= 1ull << q;

    PassRec P;
    std::memset(&P, 0, sizeof(P));
    P.k = k;
    P.c = c;
    int tile_pos[64];
    for (int q = 0; q < 64; ++q) tile_pos[q] = -1;
    {
      int j = 0;
      for (int q = 0; q < n; ++q)
        if ((Q >> q) & 1) {
          tile_pos[q] = j;
          if (j >= c) P.qhi[j - c] = q;
          ++j;
        }
      P.n_hi = k - c;
      int o = 0;
      for (int q = 0; q < n; ++q)
        if (!((Q >> q) & 1)) P.qout[o++] = q;
      P.n_out = o;
    }
    int ext_of_qubit[64];
    for (int q = 0; q < 64; ++q) ext_of_qubit[q] = -1;
    {
      const uint64_t ext = used_val & ~Q;
      int e = 0;
      for (int q = 0; q < n; ++q)
        if ((ext >> q) & 1) { ext_of_qubit[q] = e; P.ext[e] = q; ++e; }
      P.n_ext = e;
    }
    P.stage_begin = int(out->stages.size());

    // ---- stages within the pass ----
    // Virtual-index mask of a qubit read as a value (tile bit or ext bit).
    auto vmask_of = [&](int q) -> uint32_t {
      return tile_pos[q] >= 0 ? (1u << tile_pos[q]) : (1u << (k + ext_of_qubit[q]));
    };
    std::vector<int> pending = taken;
    int pass_stages = 0;
    while (!pending.empty()) {
      if (pass_stages == kMaxPassStages) {
        // stage cap reached: the ops not yet placed go back, in circuit
        // order, ahead of the ops this pass left out (they commute with every
        // earlier left-out op, or they would not have been taken)
        std::sort(pending.begin(), pending.end());
        std::vector<int> merged;
        merged.reserve(pending.size() + rest.size());
        std::merge(pending.begin(), pending.end(), rest.begin(), rest.end(), std::back_inserter(merged));
        rest.swap(merged);
        pending.clear();
        break;
      }
      ++pass_stages;
      uint64_t R = 0;          // tile-bit mask of free register bits
      uint64_t no_reg = 0;     // tile bits that must stay thread-level in this stage
      uint64_t sblocked = 0;   // qubits blocked for the rest of the stage
      uint64_t perm_q = 0;     // qubits touched by deferred permutation ops
      int n_cond = 0;
      std::vector<int> sops, sdef, srest;
      auto reg_tile_bit = [&](int q) -> int {  // tile bit of a register-capable qubit or -1
        const int tb = tile_pos[q];
        return tb;
      };
      for (int idx : pending) {
        const Op& o = ops[idx];
        const uint64_t qm = o.qubit_mask();
        if (qm & sblocked) { sblocked |= qm; srest.push_back(idx); continue; }
        uint64_t need = 0;
        const uint64_t dt_ = dense_targets(o);
        bool bad = false;
        for (int q = 0; q < n; ++q)
          if ((dt_ >> q) & 1) {
            const int tb = reg_tile_bit(q);
            if (vb == 1 && tb == 0) continue;  // complex64: tile bit 0 is always in registers
            if ((no_reg >> tb) & 1) bad = true;
            need |= 1ull << tb;
          }
        const bool fits = !bad && popc(R | need) <= kRegFree;
        // deferrable permutation: X/CNOT with <= 1 control, SWAP without controls
        bool deferrable = false;
        bool cond_ctrl = false;
        if (fits && ((o.kind == OP_X1 && o.nctrl <= 1) || (o.kind == OP_SW && o.nctrl == 0))) {
          deferrable = true;
          auto on_bit0 = [&](int q) { return vb == 1 && tile_pos[q] == 0; };
          if (o.kind == OP_X1 && o.nctrl == 1) {
            const int cq = o.ctrl[0];
            const int ctb = tile_pos[cq];
            if (on_bit0(cq) || (ctb >= 0 && (((R | need) >> ctb) & 1))) {
              cond_ctrl = false;  // register control
            } else if (ctb >= 0 && !((no_reg >> ctb) & 1) && popc(R | need | (1ull << ctb)) <= kRegFree) {
              need |= 1ull << ctb;  // room left: make the control a register bit
              cond_ctrl = false;
            } else {
              cond_ctrl = true;  // thread-level control (only once the register set is full)
            }
            if (cond_ctrl && n_cond >= kMaxCondPerm) deferrable = false;
          }
        }
        if (!fits || ((qm & perm_q) && !deferrable)) {
          sblocked |= qm;
          srest.push_back(idx);
          continue;
        }
        R |= need;
        if (deferrable) {
          sdef.push_back(idx);
          perm_q |= qm;
          if (cond_ctrl) {
            ++n_cond;
            const int ctb = tile_pos[o.ctrl[0]];
            if (ctb >= 0) no_reg |= 1ull << ctb;
          }
        } else {
          sops.push_back(idx);
        }
      }
      // fill R to exactly kRegFree tile bits (never tile bit 0 for complex64,
      // never a bit a deferred permutation reads as a thread-level control)
      for (int tb = vb; tb < k && popc(R) < kRegFree; ++tb)
        if (!((no_reg >> tb) & 1)) R |= 1ull << tb;
      if (popc(R) != kRegFree) {
        if (err) *err = "planner could not fill the register bits of a stage";
        return false;
      }
      StageRec S;
      std::memset(&S, 0, sizeof(S));
      int reg_of_tile[64];
      for (int i = 0; i < 64; ++i) reg_of_tile[i] = -1;
      if (vb == 1) reg_of_tile[0] = 0;
      {
        int j = 0;
        for (int tb = 0; tb < k; ++tb)
          if ((R >> tb) & 1) { S.rpos[j] = tb; reg_of_tile[tb] = vb + j; ++j; }
      }
      // compose the deferred permutations (in order) into pi = A p ^ b ^ conds
      {
        const int nr = vb + kRegFree;
        int a[5], b = 0;
        int cw[kMaxCondPerm];
        uint32_t cc[kMaxCondPerm];
        int nc = 0;
        for (int j = 0; j < 5; ++j) a[j] = (j < nr) ? (1 << j) : 0;
        auto apply_lin = [&](auto&& G) {
          for (int j = 0; j < nr; ++j) a[j] = G(a[j]);
          b = G(b);
          for (int i = 0; i < nc; ++i) cw[i] = G(cw[i]);
        };
        for (int idx : sdef) {
          const Op& o = ops[idx];
          const int t = reg_of_tile[tile_pos[o.t0]];
          if (o.kind == OP_SW) {
            const int u = reg_of_tile[tile_pos[o.t1]];
            apply_lin([&](int v) {
              const int bt = (v >> t) & 1, bu = (v >> u) & 1;
              return (v & ~((1 << t) | (1 << u))) | (bt << u) | (bu << t);
            });
          } else if (o.nctrl == 0) {
            b ^= 1 << t;
          } else {
            const int cq = o.ctrl[0];
            const int ctb = tile_pos[cq];
            if (ctb >= 0 && reg_of_tile[ctb] >= 0) {
              const int c = reg_of_tile[ctb];
              apply_lin([&](int v) { return v ^ (((v >> c) & 1) << t); });
            } else {
              cc[nc] = vmask_of(cq);
              cw[nc] = 1 << t;
              ++nc;
            }
          }
        }
        for (int j = 0; j < 5; ++j) S.scol[j] = a[j];
        S.sbx = b;
        S.ncond = nc;
        for (int i = 0; i < nc; ++i) { S.cond_cnr[i] = cc[i]; S.cond_w[i] = cw[i]; }
      }
      // thread-index bits: the non-register vector bits; the three lowest
      // thread bits take vector bits of distinct residue mod 3 when possible.
      std::vector<int> free_v;
      for (int tb = vb; tb < k; ++tb)
        if (!((R >> tb) & 1)) free_v.push_back(tb - vb);
      std::vector<int> order;
      for (int r = 0; r < 3; ++r) {
        for (size_t i = 0; i < free_v.size(); ++i)
          if (free_v[i] >= 0 && free_v[i] % 3 == r) { order.push_back(free_v[i]); free_v[i] = -1; break; }
      }
      for (int v : free_v)
        if (v >= 0) order.push_back(v);
      S.n_tbits = int(order.size());
      for (size_t i = 0; i < order.size(); ++i) S.tpos[i] = order[i];
      S.op_begin = int(dt == DType::C64 ? out->ops_f.size() : out->ops_d.size());
      for (int idx : sops) {
        if (dt == DType::C64)
          out->ops_f.push_back(encode_op<float>(ops[idx], tile_pos, reg_of_tile, ext_of_qubit, k));
        else
          out->ops_d.push_back(encode_op<double>(ops[idx], tile_pos, reg_of_tile, ext_of_qubit, k));
      }
      S.op_end = int(dt == DType::C64 ? out->ops_f.size() : out->ops_d.size());
      out->stages.push_back(S);
      pending.swap(srest);
    }
    P.stage_end = int(out->stages.size());
    out->passes.push_back(P);
    if (taken.empty()) {
      if (err) *err = "planner made no progress";
      return false;
    }
    remaining.swap(rest);
  }
  // Validate every table entry the kernel turns into a shift or an index.
  for (const PassRec& P : out->passes) {
    if (P.k < vb + kRegFree || P.k > kmax || P.c < 1 || P.c > P.k || P.k - P.c > 10 ||
        P.n_out != n - P.k || P.k + P.n_ext > 32) {
      if (err) *err = "invalid pass record";
      return false;
    }
    for (int si = P.stage_begin; si < P.stage_end; ++si) {
      const StageRec& S = out->stages[si];
      uint32_t used = 0;
      for (int j = 0; j < kRegFree; ++j) {
        if (S.rpos[j] < vb || S.rpos[j] >= P.k) { if (err) *err = "invalid register bit"; return false; }
        used |= 1u << (S.rpos[j] - vb);
      }
      if (S.n_tbits != P.k - vb - kRegFree) { if (err) *err = "invalid thread bits"; return false; }
      for (int j = 0; j < S.n_tbits; ++j) {
        if (S.tpos[j] < 0 || S.tpos[j] >= P.k - vb || ((used >> S.tpos[j]) & 1)) {
          if (err) *err = "invalid thread bit position";
          return false;
        }
        used |= 1u << S.tpos[j];
      }
      if (S.ncond < 0 || S.ncond > kMaxCondPerm) { if (err) *err = "invalid stage map"; return false; }
    }
  }
  out->stats.passes = out->passes.size();
  out->stats.ops = ops.size();
  out->stats.stages = out->stages.size();
  out->stats.upload_bytes = out->passes.size() * sizeof(PassRec) + out->stages.size() * sizeof(StageRec) +
                            out->ops_f.size() * sizeof(TileOp<float>) + out->ops_d.size() * sizeof(TileOp<double>);
  return true;
}

}  // namespace nqpu
