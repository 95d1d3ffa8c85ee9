// Host fusion pass of the fused (precision) mode.
//
// Generalises the reference's fuse_gates (circuits/synthesis/gate_fusion.rs:537:
// 1q runs -> 2x2, absorption of pending 1q gates into a 2q gate -> 4x4) from 2
// to 5 qubits: ops are taken greedily in circuit order while the union of
// their qubits stays within 5; an op may move ahead of an op deferred to a
// later cluster only when the two share no qubit (they commute).  Each
// cluster's 32x32 unitary is accumulated in FP64 by applying the cluster's ops
// to the 32 basis columns, with the same per-op arithmetic as the engine.
#include "fusion.h"
#include <utility>

namespace nqpu {

// Apply a lowered op to a 32-dim vector whose bit i is qubit q[i].
void fusion_apply_local(const Op& o, const int* q, cplx* v) {
  auto loc = [&](int qubit) {
    for (int i = 0; i < 5; ++i)
      if (q[i] == qubit) return i;
    return -1;
  };
  uint32_t cm = 0;
  for (int i = 0; i < o.nctrl; ++i) cm |= 1u << loc(o.ctrl[i]);
  auto ok = [&](uint32_t idx) { return (idx & cm) == cm; };
  const int b0 = o.t0 >= 0 ? loc(o.t0) : -1;
  const int b1 = o.t1 >= 0 ? loc(o.t1) : -1;
  switch (o.kind) {
    case OP_U1:
      for (uint32_t i = 0; i < 32; ++i)
        if (!((i >> b0) & 1) && ok(i)) {
          const uint32_t j = i | (1u << b0);
          const cplx x = v[i], y = v[j];
          v[i] = o.m[0] * x + o.m[1] * y;
          v[j] = o.m[2] * x + o.m[3] * y;
        }
      break;
    case OP_X1:
      for (uint32_t i = 0; i < 32; ++i)
        if (!((i >> b0) & 1) && ok(i)) std::swap(v[i], v[i | (1u << b0)]);
      break;
    case OP_PH:
      for (uint32_t i = 0; i < 32; ++i)
        if (((i >> b0) & 1) && ok(i)) v[i] *= o.m[0];
      break;
    case OP_D1:
      for (uint32_t i = 0; i < 32; ++i)
        if (ok(i)) v[i] *= o.m[(i >> b0) & 1];
      break;
    case OP_D2:
      for (uint32_t i = 0; i < 32; ++i)
        if (ok(i)) v[i] *= o.m[((i >> b1) & 1) * 2 + ((i >> b0) & 1)];
      break;
    case OP_U2:
      for (uint32_t i = 0; i < 32; ++i)
        if (!((i >> b0) & 1) && !((i >> b1) & 1) && ok(i)) {
          const uint32_t id[4] = {i, i | (1u << b0), i | (1u << b1), i | (1u << b0) | (1u << b1)};
          const cplx x[4] = {v[id[0]], v[id[1]], v[id[2]], v[id[3]]};
          for (int r = 0; r < 4; ++r)
            v[id[r]] = o.m[r * 4] * x[0] + o.m[r * 4 + 1] * x[1] + o.m[r * 4 + 2] * x[2] + o.m[r * 4 + 3] * x[3];
        }
      break;
    case OP_SW:
      for (uint32_t i = 0; i < 32; ++i)
        if (!((i >> b0) & 1) && !((i >> b1) & 1) && ok(i)) std::swap(v[i | (1u << b0)], v[i | (1u << b1)]);
      break;
    default:
      break;
  }
}

std::vector<FusedGate> fuse_ops(const std::vector<Op>& ops, int n) {
  std::vector<FusedGate> out;
  std::vector<int> pending(ops.size());
  for (size_t i = 0; i < ops.size(); ++i) pending[i] = int(i);
  while (!pending.empty()) {
    uint64_t F = 0, blocked = 0;
    std::vector<int> take, rest;
    for (int idx : pending) {
      const uint64_t qm = ops[idx].qubit_mask();
      if (qm & blocked) { blocked |= qm; rest.push_back(idx); continue; }
      if (__builtin_popcountll(F | qm) <= 5) {
        F |= qm;
        take.push_back(idx);
      } else {
        blocked |= qm;
        rest.push_back(idx);
      }
    }
    // pad to exactly 5 qubits (lowest unused qubits)
    for (int q = 0; q < n && __builtin_popcountll(F) < 5; ++q) F |= 1ull << q;
    FusedGate g;
    int j = 0;
    for (int q = 0; q < n; ++q)
      if ((F >> q) & 1) g.q[j++] = q;
    g.u.assign(32 * 32, cplx(0, 0));
    for (int c = 0; c < 32; ++c) {
      cplx col[32];
      for (int r = 0; r < 32; ++r) col[r] = (r == c) ? cplx(1, 0) : cplx(0, 0);
      for (int idx : take) fusion_apply_local(ops[idx], g.q, col);
      for (int r = 0; r < 32; ++r) g.u[r * 32 + c] = col[r];
    }
    g.n_ops = int(take.size());
    out.push_back(std::move(g));
    pending.swap(rest);
  }
  return out;
}


}  // namespace nqpu
