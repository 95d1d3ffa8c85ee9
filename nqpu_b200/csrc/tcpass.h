// Tensor-core pass mode: the plan data shared by the host planner
// (tcplan.cpp), the sm_100a kernel (tcpass.cu) and the CPU emulator of the
// kernel's index arithmetic (tests/tc_emulator.cpp).  Plain C++.
//
// One HBM pass streams the complex64 state through the SMs once.  A tile is
// the 2^12 amplitudes that agree on every qubit outside the pass's tile-qubit
// set Q (12 qubits; tile bit b <-> qubit qt[b]; tile bits 0..3 are qubits 0..3,
// so a tile is 256 runs of 16 contiguous amplitudes: 128-byte lines).  The
// pass applies up to
// kTcMaxUnitaries fused unitaries, each a dense 32x32 matrix on 5 of the tile
// qubits, in order.  For unitary j the tile is a 128 x 32 complex matrix: row
// bits = the 7 other tile bits (frow[i] = tile bit of row bit i), column bits =
// the 5 fused tile bits (fcol[i]); the contraction is one tensor-core GEMM on
// the real embedding (128 x 64 times 64 x 64).  Operands are FP16 hi/lo pairs
// (x = hi + lo, 22 significant bits) of the amplitudes scaled by a power of two
// and of 16 U, accumulated in FP32.  The tile never returns to a natural layout
// between unitaries: the epilogue of unitary j writes each amplitude straight
// to its place in unitary j+1's operand.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>
#include "sv_types.h"

namespace nqpu {

constexpr int kTcTileBits = 12;
constexpr int kTcLowBits = 4;        // tile bits 0..3 = index bits 0..3 (the 128-byte runs)
constexpr int kTcMaxUnitaries = 3;   // per pass (their B operands stay in shared memory)
constexpr int kTcMinQubits = 12;
constexpr int kTcLoadThreadBits = 7; // loading threads per tile engine: 128
constexpr int kTcLoadStepBits = 4;   // 16-byte chunks per thread: 16
constexpr int kTcMaxLaneSwaps = 2;  // last epilogue: lane exchanges with column bits 1..kTcMaxLaneSwaps
// The unitaries are stored as 16 U (entries up to 16 in magnitude keep their
// small entries clear of the FP16 subnormal range); epilogues divide by 16.
constexpr float kTcUScale = 16.0f;

// Byte offset of element (row r, 16-bit column k < 64) in a K-major operand
// with the 128-byte swizzle: 128 bytes per row (one K-atom of 64 halves),
// 8-row groups 1024 B apart, 16-byte chunks XOR-swizzled with the row within
// its group.  GF(2)-linear in the bits of (r, k), since its fields occupy
// disjoint bits.  Complex column c of a row is the half pair (re, im) at
// k = 2c, 2c + 1: 4 bytes.
inline constexpr uint32_t tc_sw128_off(uint32_t r, uint32_t k) {
  return (r >> 3) * 1024u + (r & 7u) * 128u + ((((k & 63u) * 2u >> 4) ^ (r & 7u)) << 4) + ((k & 63u) * 2u & 15u);
}

struct TcUnitaryRec {
  int32_t frow[7];      // tile bit of row bit i
  int32_t fcol[5];      // tile bit of column bit i
  uint32_t boff[12];    // A-operand byte offset contributed by tile bit b in this layout
  // Epilogue tables, per complex column c (tile part ct = deposit of c over fcol):
  uint32_t xnext[32];   // operand byte offset of ct in the NEXT unitary's layout (not the last unitary)
  uint64_t gcol[32];    // amplitude offset of ct (the last unitary: the HBM store)
};

struct TcPassRec {
  int32_t m;                     // unitaries in this pass (1..kTcMaxUnitaries)
  int32_t qt[kTcTileBits];       // state index bit of tile bit b when the pass loads (0..3: bits 0..3)
  int32_t qt_out[kTcTileBits];   // state index bit of tile bit b when the pass stores (a permutation
                                 // of qt: the pass may move qubits between index bits, see TcPlan)
  int32_t n_out;                 // qubits outside Q (tile-id bits)
  int32_t qout[kMaxQubits];      // qubit of tile-id bit j, ascending
  // loader: tile bit of loading-thread bit b (b < kTcLoadThreadBits; bits 0..2
  // are tile bits 1..3, so 8 lanes read 128 contiguous bytes) and of load-step
  // bit b - kTcLoadThreadBits; tile bit 0 is the pair inside each 16-byte load
  int32_t lt[11];
  // last epilogue: lane (row) bit exchanged with column bit 1 + s of the last
  // unitary by a shuffle before the HBM stores, or -1 (see tc_store_bits)
  int32_t sw_lane[3];
  // loader: byte offset in the operand buffer where the 16-byte raw chunk of
  // a load lands, as the XOR of one entry per tile bit (entry 0 unused: tile
  // bit 0 is the pair inside a chunk); see tc_raw_offsets
  uint32_t roff[kTcTileBits];
  TcUnitaryRec u[kTcMaxUnitaries];
};

// Raw landing offsets of a pass (TcPassRec::roff), given unitary 0's row
// order (frow0) and the loader map (lt).  The copies of a tile land as raw
// FP32 in the buffer that its FP16 hi / lo operand then overwrites, and the
// split converts it in two halves (load-step bit 3 = 0, then 1), holding only
// half the raw chunks in registers.  So the chunks of each half must land in
// the 16-byte slots that only this half's own outputs fill.  In the swizzled
// K-major layout, slot index bit i + 3 is the tile bit on row bit i (i >= 2)
// and no other tile bit's slot offset carries it, so with the half bit lt[10]
// on row bit hr (2..6) of unitary 0 the slots of half h are those with slot
// bit hr + 3 = h.  The landing is a permutation of slot bits: loading-thread
// bits 0..4 -> slot bits 0..4 (a warp's 32 chunks fill 512 contiguous bytes,
// as the copies arrive), the half bit -> slot bit hr + 3, the other chunk bits
// -> the remaining slot bits 5..10 in order.  Returns false when lt[10] is
// not on row bits 2..6 (the planner's layout choice ensures it is).
inline bool tc_raw_offsets(const int32_t* frow0, const int32_t* lt, uint32_t* roff) {
  int hr = -1;
  for (int i = 2; i < 7; ++i)
    if (frow0[i] == lt[10]) hr = i;
  if (hr < 0) return false;
  const int fbit = hr + 3;
  for (int b = 0; b < 12; ++b) roff[b] = 0;
  for (int k = 0; k < 5; ++k) roff[lt[k]] = 16u << k;
  int next = 5;
  for (int k = 5; k < 10; ++k) {
    if (next == fbit) ++next;
    roff[lt[k]] = 16u << next;
    ++next;
  }
  roff[lt[10]] = 16u << fbit;
  return true;
}

// State index bit that row bit i / column bit i of the last unitary stores to.
// The last epilogue holds D one row per lane; before its HBM stores, swap s
// exchanges lane bit sw_lane[s] with column bit 1 + s across the warp (lane
// l's register for column c then holds the amplitude of row l with that bit
// set to c's bit, column c with that bit set to l's), so that the low index
// bits of the state lie on lanes and each warp store covers whole 128-byte
// lines.  In the address tables this is the exchange of the two bits' entries.
inline void tc_store_bits(const TcPassRec& P, int32_t* row_bits, int32_t* col_bits) {
  const TcUnitaryRec& U = P.u[P.m - 1];
  for (int i = 0; i < 7; ++i) row_bits[i] = P.qt_out[U.frow[i]];
  for (int i = 0; i < 5; ++i) col_bits[i] = P.qt_out[U.fcol[i]];
  for (int s = 0; s < 3; ++s)
    if (P.sw_lane[s] >= 0) {
      const int32_t t = row_bits[P.sw_lane[s]];
      row_bits[P.sw_lane[s]] = col_bits[1 + s];
      col_bits[1 + s] = t;
    }
}

// Qubit placement: a pass may store its tile with its qubits on other state
// index bits than it loaded them from (qt_out), so that the qubits the next
// pass needs sit on index bits 0..3, which every tile must contain (they make
// the 128-byte runs of its HBM accesses).  Placements are swaps of a qubit on
// bits 0..3 with one elsewhere; the plan's last pass (or an added pass with an
// identity unitary) puts every qubit back on its own bit, so a run ends in
// the natural order.
struct TcPlan {
  int n = 0;
  float state_scale = 1.0f;      // amplitudes enter the operands multiplied by this power of two
  std::vector<TcPassRec> passes;
  // per pass, per unitary: 128 x 64 halves (as uint16 bit patterns), rows [n][k]:
  // rows 0..63 = hi, rows 64..127 = lo of the real embedding R of 16 U
  // (R[2c'+a][2c+b] = [[Re,-Im],[Im,Re]][a][b] of 16 U[c'][c])
  std::vector<uint16_t> bmats;
  // per pass, per unitary: the fused 32x32 complex unitary in FP64 (column index
  // = fcol bits), for the CPU emulator and tests
  std::vector<std::vector<cplx>> unitaries;
  // per pass: the qubit of each tile bit (the ops' qubit numbering)
  std::vector<std::array<int32_t, kTcTileBits>> lq;
  PlanStats stats;
};

constexpr size_t kTcBmatHalves = 128 * 64;

// IEEE binary16 round-to-nearest-even of a float (host side), and back.
uint16_t tc_half_bits(float x);
float tc_half_value(uint16_t h);

// Power-of-two scale of the amplitudes of an n-qubit state inside the
// operands: 2^min(max(n/2 - 2, 0), 12), so a normalised state's amplitudes
// (at most 1) stay below 2^12 and typical ones (2^(-n/2)) near 1/4.
float tc_state_scale(int n);

// Plan a lowered op list for the tensor-core pass mode (complex64, n >= 12).
// With finish = false only the pass and unitary structure is built (stats,
// pass qubits and clusters), not the layouts, offset tables or B operands.
bool build_tc_plan(const std::vector<Op>& ops, int n, TcPlan* out, std::string* err, bool finish = true);

}  // namespace nqpu
