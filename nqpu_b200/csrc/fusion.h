// Host fusion pass of the fused (precision) mode: packs runs of gates into
// dense <=5-qubit unitaries.  Plain C++ so it can be tested without a GPU.
#pragma once
#include <vector>
#include "sv_types.h"

namespace nqpu {

struct FusedGate {
  int q[5];                  // qubits, ascending; local bit i <-> q[i]
  std::vector<cplx> u;       // 32x32 row-major, FP64
  int n_ops = 0;             // original ops absorbed
};

// Greedy fusion in circuit order (see fusion.cpp); every cluster acts on
// exactly 5 qubits (padded with the lowest unused qubits).  n >= 5.
std::vector<FusedGate> fuse_ops(const std::vector<Op>& ops, int n);

// Apply a lowered op to a 32-dim vector whose bit i is qubit q[i] (every
// qubit of the op must be among q[0..4]); FP64, the engine's per-op arithmetic.
void fusion_apply_local(const Op& o, const int* q, cplx* v);

}  // namespace nqpu
