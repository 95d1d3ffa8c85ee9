// Shared plain-data types of the statevector engine: the lowered gate ("op"),
// the tiled-pass plan tables that the pass kernel reads from HBM, and the
// kernel entry points the host planner calls.  Plain C++ (no torch, no CUDA
// headers) so the planner can be compiled and unit-tested on its own.
//
// State layout in HBM (same as the reference's Vec<Complex64>, R/lib.rs:326):
// an array of 2^n complex amplitudes, interleaved (re, im), index bit q is the
// state of qubit q (LSB = qubit 0).  complex128 = 16 B/amp, complex64 = 8 B/amp.
#pragma once
#include <cstdint>
#include <complex>
#include <vector>

namespace nqpu {

using cplx = std::complex<double>;

enum class DType : int { C128 = 0, C64 = 1 };

inline int amp_bytes(DType d) { return d == DType::C128 ? 16 : 8; }

// Lowered op kinds.  Every reference gate (GateType, R/core/gates/gates.rs:8)
// lowers to one of these with optional control qubits (all controls must be 1).
enum OpKind : uint8_t {
  OP_U1 = 0,  // dense 2x2 on t0:              m[0..3] = m00 m01 m10 m11
  OP_D1 = 1,  // diag(d0, d1) on t0:           m[0..1]
  OP_X1 = 2,  // Pauli X on t0 (CNOT, Toffoli)
  OP_U2 = 3,  // dense 4x4 on (t0, t1):        m[r*4+c], sub-index = b(t1)*2 + b(t0)
  OP_D2 = 4,  // diag on (t0, t1):             m[b(t1)*2 + b(t0)]
  OP_SW = 5,  // swap t0 <-> t1 (SWAP, CSWAP)
  OP_PH = 6,  // phase m[0] on amplitudes whose bits t0 (and controls) are all 1
};

struct Op {
  uint8_t kind = OP_U1;
  uint8_t nctrl = 0;
  int8_t t0 = -1, t1 = -1;
  int8_t ctrl[3] = {-1, -1, -1};
  cplx m[16];

  // Qubits that must be addressable as a register bit to apply the op in a
  // tiled stage (dense targets).  Diagonal/phase ops and controls only need the
  // bit value, which any thread can compute from the amplitude index.
  int n_targets() const {
    switch (kind) {
      case OP_U1: case OP_X1: return 1;
      case OP_U2: case OP_SW: return 2;
      default: return 0;
    }
  }
  int target(int i) const { return i == 0 ? t0 : t1; }
  // All qubits the op reads or writes (targets, diagonal qubits, controls).
  uint64_t qubit_mask() const {
    uint64_t m_ = 0;
    if (t0 >= 0) m_ |= 1ull << t0;
    if (t1 >= 0) m_ |= 1ull << t1;
    for (int i = 0; i < nctrl; ++i) m_ |= 1ull << ctrl[i];
    return m_;
  }
  uint64_t ctrl_mask() const {
    uint64_t m_ = 0;
    for (int i = 0; i < nctrl; ++i) m_ |= 1ull << ctrl[i];
    return m_;
  }
  bool diagonal() const { return kind == OP_D1 || kind == OP_D2 || kind == OP_PH; }
};

// ----------------------------------------------------------------------------
// Tiled pass plan (consumed by the pass kernel).
//
// A pass streams the whole state through shared memory once.  A tile is the
// set of 2^k amplitudes whose indices agree on every qubit outside the pass's
// tile-qubit set Q (|Q| = k).  Q always holds qubits 0..c-1 so that a tile is
// made of 2^(k-c) contiguous runs of 2^c amplitudes (coalesced 128-bit loads).
// Inside the tile, gates run in "stages": each thread holds a register block of
// amplitudes that differ in R register bits (tile-local positions), applies all
// of the stage's ops in registers, and writes them back to shared memory.
//
// Virtual index of an amplitude: bits [0,k) = its tile-local index, bits
// [k, k+n_ext) = the values of the pass's "ext" qubits (qubits outside Q that
// some op of the pass uses as a control or diagonal qubit), constant per tile.
// ----------------------------------------------------------------------------
constexpr int kMaxQubits = 34;
constexpr int kRegFree = 4;   // free register bits per stage (plus bit 0 for complex64)

struct PassRec {
  int32_t k;                 // tile bits
  int32_t c;                 // contiguous low bits (Q[0..c-1] = 0..c-1)
  int32_t n_hi;              // k - c
  int32_t qhi[kMaxQubits];   // qubit of tile bit c+j
  int32_t n_out;             // n - k
  int32_t qout[kMaxQubits];  // qubits outside Q, ascending (tile id bit j -> qout[j])
  int32_t n_ext;
  int32_t ext[32];           // qubit of virtual bit k+j
  int32_t stage_begin, stage_end;
  int32_t pad[2];
};

// Permutation ops (X, CNOT with at most one control, SWAP) are not executed in
// registers: the planner composes them into an affine map over the register
// index bits, pi(p) = A p ^ b ^ (conditional translations), and the stage's
// write-back stores register p at the shared-memory slot of logical index
// pi(p).  scol[j] = A e_j (mask over register bits); sbx = static b;
// conditional translation i applies w = cond_w[i] when the amplitude's virtual
// index has all bits cond_cnr[i] set (a control outside the register bits).
constexpr int kMaxCondPerm = 4;
// Stages per pass are capped so that the kernels can keep every stage's
// derived constants of a pass in shared memory (kStageTabWords words each).
constexpr int kMaxPassStages = 48;
constexpr int kStageTabWords = 96;

struct StageRec {
  int32_t rpos[kRegFree];    // tile-local bit positions of the free register bits
  int32_t n_tbits;           // thread-index bits in use
  int32_t tpos[24];          // tile-local VECTOR bit position of thread-index bit j
  int32_t op_begin, op_end;  // range in the op table
  int32_t pad;
  int32_t scol[5];
  int32_t sbx;
  int32_t ncond;
  uint32_t cond_cnr[kMaxCondPerm];
  int32_t cond_w[kMaxCondPerm];
  int32_t pad2;
};

// Device op of a stage.  Register-bit numbering: complex64 register bit 0 is
// tile bit 0 (both amplitudes of a 16-byte vector), register bits 1..4 are
// rpos[0..3]; complex128 register bits 0..3 are rpos[0..3].
template <typename Real>
struct TileOp {
  uint8_t kind;
  uint8_t rb0, rb1;     // register target bits (dense ops)
  uint8_t creg;         // mask over register bits: controls held in registers
  uint8_t dreg0, dreg1; // register bit of diagonal qubit 0/1, 0xFF when not a register bit
  uint8_t fast;         // flat dispatch code of the common cases (0: decode the fields)
  uint8_t fast2;        // flat dispatch code of the diagonal shapes (read by the batch executor)
  uint32_t cnr;         // virtual-index mask of controls not in registers
  uint32_t dv0, dv1;    // virtual-index mask of diagonal qubit 0/1 when not a register bit
  uint32_t pad1[3];     // header is 32 B so m[] is 16-byte aligned
  Real m[32];           // (re, im) pairs, layout per OpKind
};

struct PlanStats {
  uint64_t passes = 0, ops = 0, stages = 0, upload_bytes = 0;
};

}  // namespace nqpu
