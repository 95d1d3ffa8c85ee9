// Host-side circuit representation, gate lowering and pass planning.
#pragma once
#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>
#include "sv_types.h"

namespace nqpu {

// Circuit-level gate codes: one per GateType variant of the reference
// (R/core/gates/gates.rs:8-62) plus the C FFI's custom gates (c_ffi.rs:663-679).
enum GateCode : uint8_t {
  G_H, G_X, G_Y, G_Z, G_S, G_T, G_SX, G_RX, G_RY, G_RZ, G_P, G_U3,
  G_CX, G_CZ, G_SWAP, G_ISWAP, G_CP, G_CRX, G_CRY, G_CRZ,
  G_RZZ, G_RXX, G_RYY, G_CCX, G_CCZ, G_CSWAP,
  G_CUSTOM1, G_CUSTOM2_FFI, G_U2_LO, G_CU,
  // mid-circuit measurement (QuantumSimulator::measure_qubit, lib.rs:1835)
  // and OpenQASM reset (measure, then X when the outcome is 1): not lowered to
  // ops, they split a circuit into segments that run as separate plans
  G_MEASURE, G_RESET,
  G_COUNT
};
inline bool gate_is_mid(uint8_t code) { return code == G_MEASURE || code == G_RESET; }

// The matrix of a custom gate (CUSTOM1: 2x2 in entries 0..3; CUSTOM2_FFI and
// U2_LO: 4x4), held out of line and shared by copies of the record until one
// of them writes (copy on write).  Records of the named gates carry none: a
// null pointer that reads as zeros, so a record stays 64 bytes and circuits of
// millions of gates copy and lower cheaply.
class GateMatrix {
 public:
  cplx operator[](int i) const { return p_ ? (*p_)[size_t(i)] : cplx(0.0, 0.0); }
  cplx& operator[](int i) {
    if (!p_) p_ = std::make_shared<std::array<cplx, 16>>();
    else if (p_.use_count() > 1) p_ = std::make_shared<std::array<cplx, 16>>(*p_);
    return (*p_)[size_t(i)];
  }

 private:
  std::shared_ptr<std::array<cplx, 16>> p_;
};

struct GateRec {
  uint8_t code = G_H;
  uint8_t nq = 1;
  int32_t q[3] = {0, 0, 0};
  double p[4] = {0, 0, 0, 0};
  GateMatrix m;  // custom matrices
};

int gate_arity(uint8_t code);
bool gate_has_params(uint8_t code);
// Lower one circuit gate to an engine op (matrices built in FP64 exactly as the
// reference builds them).
Op lower_gate(const GateRec& g);
std::vector<Op> lower_circuit(const std::vector<GateRec>& gates);

// Tiled pass plan (host tables; the engine uploads them).
struct TilePlan {
  DType dt = DType::C128;
  int n = 0;
  std::vector<PassRec> passes;
  std::vector<StageRec> stages;
  std::vector<TileOp<float>> ops_f;
  std::vector<TileOp<double>> ops_d;
  PlanStats stats;
};

// Minimum qubit count the tiled kernel supports for a dtype (smaller states use
// the per-gate kernels).
int tile_min_qubits(DType dt);
// kmax: tile bits of the kernel (13 for complex64, 12 for complex128).
bool build_tile_plan(const std::vector<Op>& ops, int n, DType dt, int kmax, TilePlan* out,
                     std::string* err);

// Greedy layer depth (c_ffi.rs:697-720).
uint32_t circuit_depth(const std::vector<GateRec>& gates, uint32_t n);

}  // namespace nqpu
