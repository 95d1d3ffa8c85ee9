// Host planner of the tensor-core pass mode (see tcpass.h for the plan data).
//
// Passes: ops are taken greedily in circuit order into the current pass while
// the union of their qubits with qubits 0..4 stays within 12 (the tile); an op
// may move ahead of an op left for a later pass only when the two share no
// qubit (they commute), as in the tiled planner.  Within a pass the taken ops
// are packed greedily, in order and under the same commutation rule, into
// clusters of at most 5 qubits (the reference's fuse_gates, gate_fusion.rs:537,
// generalised from 2 to 5 qubits); at most kTcMaxUnitaries clusters per pass,
// the ops of any further cluster go back, in circuit order, ahead of the ops
// the pass left out.  Each cluster becomes one 32x32 unitary accumulated in
// FP64 with the engine's per-op arithmetic, then its real embedding is split
// into TF32 hi/lo parts for the tensor cores.
//
// Layouts: for unitary j the planner also picks which tile bits are the
// operand's row bits 0..4.  Those decide the shared-memory banks of the
// operand stores (the loader's stores into layout 0, the epilogue of unitary j
// storing into layout j+1) and the coalescing of the last epilogue's HBM
// stores; a small dynamic programme over the layouts of the pass minimises the
// store wavefronts (rank of the lane bits' address images, see store_cost).
#include "tcpass.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <iterator>

#include "fusion.h"

namespace nqpu {

namespace {

int popc(uint64_t x) { return __builtin_popcountll(x); }

uint32_t rn_tf32(float x) {
  uint32_t b;
  std::memcpy(&b, &x, 4);
  return (b + 0x1000u) & 0xFFFFE000u;
}
float as_float(uint32_t b) {
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

// Row choice of one layout: tile bits of row bits 0..4 (the remaining row bits
// follow in ascending tile-bit order).
struct RowChoice {
  int lane[5];
};

// Byte offsets of the tile bits in a layout (frow / fcol given).
void layout_offsets(const int* frow, const int* fcol, uint32_t* boff) {
  for (int i = 0; i < 7; ++i) boff[frow[i]] = tc_sw128_off<128>(1u << i, 0);
  for (int i = 0; i < 5; ++i) boff[fcol[i]] = tc_sw128_off<128>(0, 2u << i);
}

// GF(2) rank of 4-bit vectors.
int rank4(const uint32_t* v, int cnt) {
  uint32_t basis[4] = {0, 0, 0, 0};
  int r = 0;
  for (int i = 0; i < cnt; ++i) {
    uint32_t x = v[i] & 15u;
    for (int b = 3; b >= 0; --b) {
      if (!((x >> b) & 1u)) continue;
      if (!basis[b]) {
        basis[b] = x;
        ++r;
        break;
      }
      x ^= basis[b];
    }
  }
  return r;
}

// Wavefronts of an 8-byte shared-memory store by a half warp whose lanes 0..15
// run over the tile bits lb[0..3]: 2^(4 - rank) of the lanes' bank-slot bits
// (address bits 3..6) in the target layout.
int store_cost(const int* lb, const uint32_t* boff) {
  uint32_t v[4];
  for (int i = 0; i < 4; ++i) v[i] = boff[lb[i]] >> 3;
  return 1 << (4 - rank4(v, 4));
}

// 32-byte sectors of a warp's 8-byte HBM stores whose lanes run over the tile
// bits lb[0..4] (tile bits 0 and 1 are qubits 0 and 1: 4 amplitudes per
// sector), divided by the ideal 8.
int hbm_cost(const int* lb) {
  int low = 0;
  for (int i = 0; i < 5; ++i) low += (lb[i] == 0 || lb[i] == 1) ? 1 : 0;
  return 1 << (2 - low);
}

void fill_rows(const RowChoice& rc, uint32_t fmask, int* frow) {
  int j = 0;
  uint32_t used = fmask;
  for (int i = 0; i < 5; ++i) {
    frow[j++] = rc.lane[i];
    used |= 1u << rc.lane[i];
  }
  for (int b = 0; b < kTcTileBits; ++b)
    if (!((used >> b) & 1u)) frow[j++] = b;
}

// Candidate row choices of a layout: every ordered pick of 5 of the 7 row
// tile bits reduces, for the costs above, to (set of rows 0..2, row 3, row 4);
// the order inside rows 0..2 does not change any rank.
std::vector<RowChoice> candidates(uint32_t fmask) {
  int rows[7], nr = 0;
  for (int b = 0; b < kTcTileBits; ++b)
    if (!((fmask >> b) & 1u)) rows[nr++] = b;
  std::vector<RowChoice> out;
  for (int a = 0; a < 7; ++a)
    for (int b = a + 1; b < 7; ++b)
      for (int c = b + 1; c < 7; ++c)
        for (int d = 0; d < 7; ++d) {
          if (d == a || d == b || d == c) continue;
          for (int e = 0; e < 7; ++e) {
            if (e == a || e == b || e == c || e == d) continue;
            RowChoice rc;
            rc.lane[0] = rows[a];
            rc.lane[1] = rows[b];
            rc.lane[2] = rows[c];
            rc.lane[3] = rows[d];
            rc.lane[4] = rows[e];
            out.push_back(rc);
          }
        }
  return out;
}

// Choose the row layouts of a pass's unitaries (fcol fixed) by dynamic
// programming over the chain loader -> L0 -> L1 -> ... -> HBM.
void choose_layouts(TcPassRec& P) {
  const int m = P.m;
  std::vector<std::vector<RowChoice>> cand(static_cast<size_t>(m));
  std::vector<std::vector<std::array<uint32_t, 12>>> offs(static_cast<size_t>(m));
  for (int j = 0; j < m; ++j) {
    uint32_t fmask = 0;
    for (int i = 0; i < 5; ++i) fmask |= 1u << P.u[j].fcol[i];
    cand[size_t(j)] = candidates(fmask);
    for (const RowChoice& rc : cand[size_t(j)]) {
      int frow[7];
      fill_rows(rc, fmask, frow);
      std::array<uint32_t, 12> bo{};
      layout_offsets(frow, P.u[j].fcol, bo.data());
      offs[size_t(j)].push_back(bo);
    }
  }
  // the loader's half-warp lanes run over tile bits 1..4
  const int loader_lanes[4] = {1, 2, 3, 4};
  std::vector<std::vector<int>> best(static_cast<size_t>(m)), from(static_cast<size_t>(m));
  for (int j = 0; j < m; ++j) {
    const size_t nc = cand[size_t(j)].size();
    best[size_t(j)].assign(nc, 1 << 30);
    from[size_t(j)].assign(nc, -1);
    for (size_t ci = 0; ci < nc; ++ci) {
      const uint32_t* bo = offs[size_t(j)][ci].data();
      if (j == 0) {
        best[0][ci] = store_cost(loader_lanes, bo);
        continue;
      }
      for (size_t pi = 0; pi < cand[size_t(j - 1)].size(); ++pi) {
        const int c = best[size_t(j - 1)][pi] + store_cost(cand[size_t(j - 1)][pi].lane, bo);
        if (c < best[size_t(j)][ci]) {
          best[size_t(j)][ci] = c;
          from[size_t(j)][ci] = int(pi);
        }
      }
    }
  }
  // the last layout's epilogue stores to HBM (weighted as a global store)
  int bi = 0, bc = 1 << 30;
  for (size_t ci = 0; ci < cand[size_t(m - 1)].size(); ++ci) {
    const int c = best[size_t(m - 1)][ci] + 2 * hbm_cost(cand[size_t(m - 1)][ci].lane);
    if (c < bc) {
      bc = c;
      bi = int(ci);
    }
  }
  for (int j = m - 1; j >= 0; --j) {
    uint32_t fmask = 0;
    for (int i = 0; i < 5; ++i) fmask |= 1u << P.u[j].fcol[i];
    fill_rows(cand[size_t(j)][size_t(bi)], fmask, P.u[j].frow);
    bi = from[size_t(j)][size_t(bi)];
  }
}

}  // namespace

bool build_tc_plan(const std::vector<Op>& ops, int n, TcPlan* out, std::string* err) {
  out->n = n;
  out->passes.clear();
  out->bmats.clear();
  out->unitaries.clear();
  out->stats = PlanStats{};
  if (n < kTcMinQubits || n > kMaxQubits) {
    if (err) *err = "the tensor-core pass mode needs 12 <= n <= 34 qubits";
    return false;
  }
  const uint64_t low = (1ull << kTcLowBits) - 1;
  std::vector<int> remaining(ops.size());
  for (size_t i = 0; i < ops.size(); ++i) remaining[i] = int(i);
  while (!remaining.empty()) {
    // ---- ops of the pass ----
    uint64_t Q = low, blocked = 0;
    std::vector<int> taken, rest;
    for (int idx : remaining) {
      const uint64_t qm = ops[size_t(idx)].qubit_mask();
      if (qm & blocked) {
        blocked |= qm;
        rest.push_back(idx);
        continue;
      }
      if (popc(Q | qm) <= kTcTileBits) {
        Q |= qm;
        taken.push_back(idx);
      } else {
        blocked |= qm;
        rest.push_back(idx);
      }
    }
    // ---- clusters of <= 5 qubits ----
    std::vector<std::pair<uint64_t, std::vector<int>>> clusters;
    std::vector<int> pend = taken;
    while (!pend.empty() && int(clusters.size()) < kTcMaxUnitaries) {
      uint64_t F = 0, cb = 0;
      std::vector<int> cl, pr;
      for (int idx : pend) {
        const uint64_t qm = ops[size_t(idx)].qubit_mask();
        if (qm & cb) {
          cb |= qm;
          pr.push_back(idx);
          continue;
        }
        if (popc(F | qm) <= 5) {
          F |= qm;
          cl.push_back(idx);
        } else {
          cb |= qm;
          pr.push_back(idx);
        }
      }
      clusters.emplace_back(F, std::move(cl));
      pend.swap(pr);
    }
    if (!pend.empty()) {
      // ops of clusters beyond the cap go back in circuit order, ahead of the
      // ops left out of the pass (they commute with every earlier left-out op)
      std::sort(pend.begin(), pend.end());
      std::vector<int> merged;
      merged.reserve(pend.size() + rest.size());
      std::merge(pend.begin(), pend.end(), rest.begin(), rest.end(), std::back_inserter(merged));
      rest.swap(merged);
    }
    // fill the tile to 12 qubits with the lowest unused qubits
    for (int q = 0; q < n && popc(Q) < kTcTileBits; ++q) Q |= 1ull << q;

    TcPassRec P;
    std::memset(&P, 0, sizeof(P));
    P.m = int(clusters.size());
    {
      int b = 0;
      for (int q = 0; q < n; ++q)
        if ((Q >> q) & 1ull) P.qt[b++] = q;
      int o = 0;
      for (int q = 0; q < n; ++q)
        if (!((Q >> q) & 1ull)) P.qout[o++] = q;
      P.n_out = o;
    }
    for (int j = 0; j < P.m; ++j) {
      uint64_t F = clusters[size_t(j)].first;
      // pad to exactly 5 qubits with the lowest unused tile qubits
      for (int b = 0; b < kTcTileBits && popc(F) < 5; ++b) F |= 1ull << P.qt[b];
      int i = 0;
      for (int b = 0; b < kTcTileBits; ++b)
        if ((F >> P.qt[b]) & 1ull) P.u[j].fcol[i++] = b;
    }
    choose_layouts(P);
    // ---- offset tables ----
    for (int j = 0; j < P.m; ++j) layout_offsets(P.u[j].frow, P.u[j].fcol, P.u[j].boff);
    for (int j = 0; j < P.m; ++j) {
      TcUnitaryRec& U = P.u[j];
      for (uint32_t c = 0; c < 32; ++c) {
        uint32_t x = 0;
        uint64_t g = 0;
        for (int i = 0; i < 5; ++i)
          if ((c >> i) & 1u) {
            if (j + 1 < P.m) x ^= P.u[j + 1].boff[U.fcol[i]];
            g |= 1ull << P.qt[U.fcol[i]];
          }
        U.xnext[c] = x;
        U.gcol[c] = g;
      }
    }
    // ---- unitaries and their split real embeddings ----
    for (int j = 0; j < P.m; ++j) {
      int q[5];
      for (int i = 0; i < 5; ++i) q[i] = P.qt[P.u[j].fcol[i]];
      std::vector<cplx> u(32 * 32, cplx(0, 0));
      for (int c = 0; c < 32; ++c) {
        cplx col[32];
        for (int r = 0; r < 32; ++r) col[r] = (r == c) ? cplx(1, 0) : cplx(0, 0);
        for (int idx : clusters[size_t(j)].second) fusion_apply_local(ops[size_t(idx)], q, col);
        for (int r = 0; r < 32; ++r) u[size_t(r * 32 + c)] = col[r];
      }
      const size_t base = out->bmats.size();
      out->bmats.resize(base + kTcBmatFloats);
      float* B = out->bmats.data() + base;
      for (int co = 0; co < 32; ++co)
        for (int ci = 0; ci < 32; ++ci) {
          const cplx v = u[size_t(co * 32 + ci)];
          const double e[2][2] = {{v.real(), -v.imag()}, {v.imag(), v.real()}};
          for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
              const int nrow = 2 * co + a, k = 2 * ci + b;
              const float hi = as_float(rn_tf32(float(e[a][b])));
              const float lo = as_float(rn_tf32(float(e[a][b] - double(hi))));
              B[nrow * 64 + k] = hi;
              B[(64 + nrow) * 64 + k] = lo;
            }
        }
      out->unitaries.push_back(std::move(u));
    }
    out->passes.push_back(P);
    out->stats.stages += uint64_t(P.m);
    remaining.swap(rest);
  }
  out->stats.passes = out->passes.size();
  out->stats.ops = ops.size();
  out->stats.upload_bytes = out->passes.size() * sizeof(TcPassRec) + out->bmats.size() * sizeof(float);
  return true;
}

}  // namespace nqpu
