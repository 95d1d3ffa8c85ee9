// Test infrastructure: a CPU emulation of the tiled pass kernel
// (nqpu_b200/csrc/kernels_tile.cu) that executes the planner's tables
// (PassRec / StageRec / TileOp) with the kernel's index arithmetic — swizzled
// shared-memory slots, register blocks, register-bit op semantics and the
// affine write-back of deferred permutations — in FP64.  It lets the CPU test
// suite check the planner and the kernel's addressing against the oracle.
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "planner.h"
#include "fusion.h"

using namespace nqpu;
using cd = std::complex<double>;

namespace {

uint32_t swz(uint32_t u) {
  uint32_t w = u >> 3;
  uint32_t f = w ^ (w >> 3) ^ (w >> 6) ^ (w >> 9) ^ (w >> 12);
  return u ^ (f & 7u);
}

template <typename Real>
cd mget(const TileOp<Real>& op, int i) { return cd(double(op.m[2 * i]), double(op.m[2 * i + 1])); }

// Apply one encoded op to a register block of NA amplitudes (NRB register bits).
template <typename Real>
void apply_op(const TileOp<Real>& op, std::vector<cd>& a, int NRB, uint32_t vbase) {
  const int NA = 1 << NRB;
  const bool tc = (vbase & op.cnr) == op.cnr;
  auto cond = [&](int i) { return tc && ((uint32_t(i) & op.creg) == op.creg); };
  switch (op.kind) {
    case OP_U1: {
      const int B = op.rb0;
      for (int i = 0; i < NA; ++i) {
        if (i & (1 << B)) continue;
        const int j = i | (1 << B);
        if (!cond(i)) continue;
        const cd x = a[i], y = a[j];
        a[i] = mget(op, 0) * x + mget(op, 1) * y;
        a[j] = mget(op, 2) * x + mget(op, 3) * y;
      }
      break;
    }
    case OP_X1: {
      const int B = op.rb0;
      for (int i = 0; i < NA; ++i) {
        if (i & (1 << B)) continue;
        if (cond(i)) std::swap(a[i], a[i | (1 << B)]);
      }
      break;
    }
    case OP_PH:
      for (int i = 0; i < NA; ++i)
        if (cond(i)) a[i] *= mget(op, 0);
      break;
    case OP_D1:
    case OP_D2: {
      const uint32_t tb0 = (vbase & op.dv0) ? 1u : 0u, tb1 = (vbase & op.dv1) ? 1u : 0u;
      for (int i = 0; i < NA; ++i) {
        if (!cond(i)) continue;
        const uint32_t b0 = op.dreg0 != 0xFF ? ((uint32_t(i) >> op.dreg0) & 1u) : tb0;
        const uint32_t b1 = op.kind == OP_D2 ? (op.dreg1 != 0xFF ? ((uint32_t(i) >> op.dreg1) & 1u) : tb1) : 0u;
        a[i] *= mget(op, int(b1 * 2 + b0));
      }
      break;
    }
    case OP_U2: {
      const int M0 = 1 << op.rb0, M1 = 1 << op.rb1;
      for (int i = 0; i < NA; ++i) {
        if (i & (M0 | M1)) continue;
        if (!cond(i)) continue;
        const cd x[4] = {a[i], a[i | M0], a[i | M1], a[i | M0 | M1]};
        cd y[4];
        for (int r = 0; r < 4; ++r) {
          y[r] = 0;
          for (int c = 0; c < 4; ++c) y[r] += mget(op, r * 4 + c) * x[c];
        }
        a[i] = y[0]; a[i | M0] = y[1]; a[i | M1] = y[2]; a[i | M0 | M1] = y[3];
      }
      break;
    }
    case OP_SW: {
      const int M0 = 1 << op.rb0, M1 = 1 << op.rb1;
      for (int i = 0; i < NA; ++i) {
        if (i & (M0 | M1)) continue;
        if (cond(i)) std::swap(a[i | M0], a[i | M1]);
      }
      break;
    }
    default:
      break;
  }
}

template <typename Real>
void run_plan(const TilePlan& plan, std::vector<cd>& st) {
  const int VB = std::is_same<Real, float>::value ? 1 : 0;
  const int APV = 1 << VB;
  const int NRB = VB + kRegFree;
  const int kVecPerThread = 16;
  const std::vector<TileOp<Real>>& ops = *reinterpret_cast<const std::vector<TileOp<Real>>*>(
      std::is_same<Real, float>::value ? static_cast<const void*>(&plan.ops_f) : static_cast<const void*>(&plan.ops_d));
  for (const PassRec& P : plan.passes) {
    const int k = P.k, c = P.c;
    const uint32_t nvec = 1u << (k - VB);
    const uint64_t n_tiles = 1ull << P.n_out;
    std::vector<uint64_t> hi_off(1u << (k - c));
    for (uint32_t h = 0; h < hi_off.size(); ++h) {
      uint64_t off = 0;
      for (int j = 0; j < k - c; ++j)
        if ((h >> j) & 1) off |= 1ull << P.qhi[j];
      hi_off[h] = off;
    }
    const uint32_t lowmask = (1u << c) - 1u;
    const uint32_t active = nvec / kVecPerThread;
    std::vector<cd> sm(size_t(nvec) * APV);  // smem: slot-major, APV amps per slot
    for (uint64_t tile = 0; tile < n_tiles; ++tile) {
      uint64_t base = 0;
      for (int j = 0; j < P.n_out; ++j)
        if ((tile >> j) & 1ull) base |= 1ull << P.qout[j];
      uint32_t ext = 0;
      for (int j = 0; j < P.n_ext; ++j)
        if ((base >> P.ext[j]) & 1ull) ext |= 1u << (k + j);
      auto gaddr = [&](uint32_t u) {
        const uint32_t t = u << VB;
        return base + (t & lowmask) + hi_off[t >> c];
      };
      for (uint32_t u = 0; u < nvec; ++u)
        for (int h = 0; h < APV; ++h) sm[size_t(swz(u)) * APV + h] = st[gaddr(u) + h];
      for (int s = P.stage_begin; s < P.stage_end; ++s) {
        const StageRec& S = plan.stages[s];
        std::vector<cd> nsm = sm;  // threads write disjoint slots; emulate via a copy
        for (uint32_t tid = 0; tid < active; ++tid) {
          uint32_t ub = 0;
          for (int j = 0; j < S.n_tbits; ++j) ub |= ((tid >> j) & 1u) << S.tpos[j];
          const uint32_t sv[4] = {swz(1u << (S.rpos[0] - VB)), swz(1u << (S.rpos[1] - VB)),
                                  swz(1u << (S.rpos[2] - VB)), swz(1u << (S.rpos[3] - VB))};
          const uint32_t sb = swz(ub);
          auto rslot = [&](int r) {
            uint32_t x = sb;
            for (int q = 0; q < 4; ++q)
              if (r & (1 << q)) x ^= sv[q];
            return x;
          };
          std::vector<cd> a(size_t(kVecPerThread) * APV);
          for (int r = 0; r < kVecPerThread; ++r)
            for (int h = 0; h < APV; ++h) a[r * APV + h] = sm[size_t(rslot(r)) * APV + h];
          const uint32_t vbase = (ub << VB) | ext;
          for (int o = S.op_begin; o < S.op_end; ++o) apply_op<Real>(ops[o], a, NRB, vbase);
          // affine write-back
          uint32_t w = uint32_t(S.sbx);
          for (int i = 0; i < S.ncond; ++i)
            if ((vbase & S.cond_cnr[i]) == S.cond_cnr[i]) w ^= uint32_t(S.cond_w[i]);
          auto regslot = [&](uint32_t m) {
            uint32_t x = 0;
            for (int q = 0; q < 4; ++q)
              if ((m >> (VB + q)) & 1u) x ^= sv[q];
            return x;
          };
          for (int p = 0; p < kVecPerThread * APV; ++p) {
            uint32_t m = w;
            for (int j = 0; j < NRB; ++j)
              if ((p >> j) & 1) m ^= uint32_t(S.scol[j]);
            const uint32_t slot = sb ^ regslot(m);
            const int half = VB ? int(m & 1u) : 0;
            nsm[size_t(slot) * APV + half] = a[p];
          }
        }
        sm.swap(nsm);
      }
      for (uint32_t u = 0; u < nvec; ++u)
        for (int h = 0; h < APV; ++h) st[gaddr(u) + h] = sm[size_t(swz(u)) * APV + h];
    }
  }
}

}  // namespace

extern "C" int emu_run(int n, int c64, const double* flat, int ngates, double* state) {
  std::vector<GateRec> gates(ngates);
  for (int i = 0; i < ngates; ++i) {
    const double* g = flat + size_t(i) * 40;
    GateRec& r = gates[i];
    r.code = uint8_t(g[0]);
    r.nq = uint8_t(gate_arity(r.code));
    for (int j = 0; j < 3; ++j) r.q[j] = int(g[1 + j]);
    for (int j = 0; j < 4; ++j) r.p[j] = g[4 + j];
    for (int j = 0; j < 16; ++j) r.m[j] = cplx(g[8 + 2 * j], g[9 + 2 * j]);
  }
  const DType dt = c64 ? DType::C64 : DType::C128;
  TilePlan plan;
  std::string err;
  const std::vector<Op> ops = lower_circuit(gates);
  if (!build_tile_plan(ops, n, dt, c64 ? 13 : 12, &plan, &err)) return -1;
  std::vector<cd> st(size_t(1) << n);
  for (size_t i = 0; i < st.size(); ++i) st[i] = cd(state[2 * i], state[2 * i + 1]);
  if (c64) run_plan<float>(plan, st);
  else run_plan<double>(plan, st);
  for (size_t i = 0; i < st.size(); ++i) { state[2 * i] = st[i].real(); state[2 * i + 1] = st[i].imag(); }
  return int(plan.passes.size());
}

// Fusion pass check: apply the fused 32x32 unitaries in FP64.  Returns the
// number of fused unitaries.
extern "C" int emu_fused(int n, const double* flat, int ngates, double* state) {
  std::vector<GateRec> gates(ngates);
  for (int i = 0; i < ngates; ++i) {
    const double* g = flat + size_t(i) * 40;
    GateRec& r = gates[i];
    r.code = uint8_t(g[0]);
    r.nq = uint8_t(gate_arity(r.code));
    for (int j = 0; j < 3; ++j) r.q[j] = int(g[1 + j]);
    for (int j = 0; j < 4; ++j) r.p[j] = g[4 + j];
    for (int j = 0; j < 16; ++j) r.m[j] = cplx(g[8 + 2 * j], g[9 + 2 * j]);
  }
  const std::vector<FusedGate> fg = fuse_ops(lower_circuit(gates), n);
  const size_t dim = size_t(1) << n;
  std::vector<cd> st(dim);
  for (size_t i = 0; i < dim; ++i) st[i] = cd(state[2 * i], state[2 * i + 1]);
  for (const FusedGate& f : fg) {
    uint64_t fm = 0;
    for (int b = 0; b < 5; ++b) fm |= 1ull << f.q[b];
    for (size_t base = 0; base < dim; ++base) {
      if (base & fm) continue;
      cd v[32], w[32];
      for (int j = 0; j < 32; ++j) {
        size_t idx = base;
        for (int b = 0; b < 5; ++b)
          if ((j >> b) & 1) idx |= size_t(1) << f.q[b];
        v[j] = st[idx];
      }
      for (int r = 0; r < 32; ++r) {
        w[r] = 0;
        for (int c = 0; c < 32; ++c) w[r] += f.u[r * 32 + c] * v[c];
      }
      for (int j = 0; j < 32; ++j) {
        size_t idx = base;
        for (int b = 0; b < 5; ++b)
          if ((j >> b) & 1) idx |= size_t(1) << f.q[b];
        st[idx] = w[j];
      }
    }
  }
  for (size_t i = 0; i < dim; ++i) { state[2 * i] = st[i].real(); state[2 * i + 1] = st[i].imag(); }
  return int(fg.size());
}
