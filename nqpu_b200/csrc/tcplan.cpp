// Host planner of the tensor-core pass mode (see tcpass.h for the plan data).
//
// Passes: ops are taken greedily in circuit order into the current pass while
// the union of their qubits with qubits 0..3 stays within 12 (the tile); an op
// may move ahead of an op left for a later pass only when the two share no
// qubit (they commute), as in the tiled planner.  Within a pass the taken ops
// are packed greedily, in order and under the same commutation rule, into
// clusters of at most 5 qubits (the reference's fuse_gates, gate_fusion.rs:537,
// generalised from 2 to 5 qubits); at most kTcMaxUnitaries clusters per pass,
// the ops of any further cluster go back, in circuit order, ahead of the ops
// the pass left out.  Each cluster becomes one 32x32 unitary accumulated in
// FP64 with the engine's per-op arithmetic, then the real embedding of 16 U is
// split into FP16 hi/lo parts for the tensor cores.
//
// Layouts: for unitary j the planner also picks which tile bits are the
// operand's row bits 0..4.  Those decide the shared-memory banks of the
// operand stores (the loader's stores into layout 0, the epilogue of unitary j
// storing into layout j+1) and the coalescing of the last epilogue's HBM
// stores; a small dynamic programme over the layouts of the pass minimises the
// store wavefronts (rank of the lane bits' address images, see store_cost).
#include "tcpass.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <iterator>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "fusion.h"

namespace nqpu {

namespace {

int popc(uint64_t x) { return __builtin_popcountll(x); }

// Byte offsets of the tile bits in a layout (frow / fcol given).
void layout_offsets(const int* frow, const int* fcol, uint32_t* boff) {
  for (int i = 0; i < 7; ++i) boff[frow[i]] = tc_sw128_off(1u << i, 0);
  for (int i = 0; i < 5; ++i) boff[fcol[i]] = tc_sw128_off(0, 2u << i);  // complex column bit i = half 2 << i
}

// GF(2) rank of 5-bit vectors (bits above 4 ignored).
int rank5(const uint32_t* v, int cnt) {
  uint32_t basis[5] = {0, 0, 0, 0, 0};
  int r = 0;
  for (int i = 0; i < cnt; ++i) {
    uint32_t x = v[i] & 31u;
    for (int b = 4; b >= 0; --b) {
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

// Shared-memory wavefronts of one warp-wide store of `width` bytes per lane
// whose lanes run over the tile bits lb[0..4], into a layout with byte offsets
// boff.  A 4-byte store is one wavefront when the lanes' images in address
// bits 2..6 (the bank) are independent; 8-byte stores go out a half warp
// (lane bits 0..3, address bits 3..6) and 16-byte stores a quarter warp (lane
// bits 0..2, address bits 4..6) at a time.  (The kernel's ncu store-wavefront
// counts follow this rule.)
int store_wavefronts(const int* lb, const uint32_t* boff, int width) {
  uint32_t v[5];
  if (width == 16) {
    for (int i = 0; i < 3; ++i) v[i] = (boff[lb[i]] >> 4) & 7u;
    return 4 << (3 - rank5(v, 3));
  }
  if (width == 8) {
    for (int i = 0; i < 4; ++i) v[i] = (boff[lb[i]] >> 3) & 15u;
    return 2 << (4 - rank5(v, 4));
  }
  for (int i = 0; i < 5; ++i) v[i] = (boff[lb[i]] >> 2) & 31u;
  return 1 << (5 - rank5(v, 5));
}

// Lane exchanges of the last epilogue (TcPassRec::sw_lane): column bit 1 + s
// of the last unitary, when it stores to index bit 0..3, trades places with
// the free lane bit (row bits 0..4) that stores to the highest index bit >= 4.
// Each exchange halves the 128-byte lines a warp store touches (a line holds
// the 16 amplitudes that differ in index bits 0..3).  qt: store-side index
// bits of the tile bits.
int lane_swaps(const int* frow, const int* fcol, const int* qt, int32_t* sw) {
  bool used[5] = {false, false, false, false, false};
  int cnt = 0;
  int order[3] = {1, 2, 3};  // column bits by their index bit, lowest first
  std::sort(order, order + kTcMaxLaneSwaps, [&](int a, int b) { return qt[fcol[a]] < qt[fcol[b]]; });
  for (int s = 0; s < 3; ++s) sw[s] = -1;
  for (int k = 0; k < kTcMaxLaneSwaps; ++k) {
    const int cb = order[k];
    if (qt[fcol[cb]] > 3) continue;
    int best = -1;
    for (int i = 0; i < 5; ++i)
      if (!used[i] && qt[frow[i]] >= 4 && (best < 0 || qt[frow[i]] > qt[frow[best]])) best = i;
    if (best < 0) break;
    used[best] = true;
    sw[cb - 1] = best;
    ++cnt;
  }
  return cnt;
}

// Layout choice of a pass: column order and row order of every unitary's
// operand, and the loader's map from thread / step bits to tile bits.
struct LayoutCfg {
  int fcol[kTcMaxUnitaries][5];
  int frow[kTcMaxUnitaries][7];
  int lt[11];
};

// Per-tile cost of a layout choice: shared-memory store wavefronts of the
// loader and of the epilogues that feed the next unitary, plus, for the last
// epilogue's HBM stores (after its lane exchanges), a quarter unit per 32-byte
// sector and four units per 128-byte line a warp store touches beyond the
// minimum, and 256 units per lane exchange (its shuffles).  (Measured on the
// 30-qubit brickwork: stores at 4 lines per warp instead of 10-11 shorten a
// tile's last epilogue by 1000-3000 cycles.)
int layout_cost(const LayoutCfg& c, int m, const int* qt) {
  uint32_t boff[kTcMaxUnitaries][12];
  for (int j = 0; j < m; ++j) layout_offsets(c.frow[j], c.fcol[j], boff[j]);
  int cost = 0;
  // loader: 64 warp-steps per tile (4 warps x 16 steps), lanes over tile
  // bits lt[0..4], hi and lo
  // planes; the two amplitudes of a 16-byte load are one 8-byte store when
  // tile bit 0 is column bit 0 of unitary 0, else two 4-byte stores
  if (c.fcol[0][0] == 0) cost += 64 * 2 * store_wavefronts(c.lt, boff[0], 8);
  else cost += 64 * 2 * 2 * store_wavefronts(c.lt, boff[0], 4);
  // the split's half bit lt[10] must sit on row bits 2..6 of unitary 0 (the
  // raw landing offsets need it; any other choice is invalid)
  uint32_t roff[kTcTileBits];
  if (!tc_raw_offsets(c.frow[0], c.lt, roff)) return 1 << 24;
  // epilogue: 4 warps x 32 columns (128 column-stores per tile, or 256
  // single ones), pairs of columns as 8-byte stores when
  // both layouts share column bit 0
  for (int j = 0; j + 1 < m; ++j) {
    const bool pair = c.fcol[j][0] == c.fcol[j + 1][0];
    cost += 4 * (pair ? 16 : 32) * 2 * store_wavefronts(c.frow[j], boff[j + 1], pair ? 8 : 4);
  }
  // HBM: lanes over rows 0..4 of the last layout, after the lane exchanges.
  // A warp store touches 2^k sectors (32 bytes: index bits 0, 1 inside) when k
  // lane bits store to index bits >= 2, and 2^k' lines when k' of them store
  // to index bits >= 4; the minima are 16 sectors / 4 lines for 16-byte
  // stores (index bit 0 is column bit 0 and each lane writes a pair) and 8 / 2
  // for 8-byte ones.
  const int L = m - 1;
  const bool wide = qt[c.fcol[L][0]] == 0;  // qt: the store-side index bits (qt_out)
  int32_t sw[3];
  const int nsw = lane_swaps(c.frow[L], c.fcol[L], qt, sw);
  int lane_bit[5];
  for (int i = 0; i < 5; ++i) lane_bit[i] = qt[c.frow[L][i]];
  for (int s = 0; s < 3; ++s)
    if (sw[s] >= 0) lane_bit[sw[s]] = qt[c.fcol[L][1 + s]];
  int ks = 0, kl = 0;
  for (int i = 0; i < 5; ++i) {
    ks += lane_bit[i] >= 2 ? 1 : 0;
    kl += lane_bit[i] >= 4 ? 1 : 0;
  }
  const int instr = 4 * (wide ? 16 : 32);
  cost += instr * (((1 << ks) - (wide ? 16 : 8)) / 4 + 4 * ((1 << kl) - (wide ? 4 : 2))) + 256 * nsw;
  return cost;
}

// Deterministic local search (best-improvement swaps from the sorted layout,
// then seeded restarts until the cost reaches its lower bound) for the layout
// choice of a pass.  The cost depends only on m and the fused tile-bit sets,
// so results are kept in a process-wide cache keyed by those.
std::mutex g_layout_mu;
std::unordered_map<uint64_t, LayoutCfg> g_layout_cache;

void choose_layouts(TcPassRec& P) {
  const int m = P.m;
  uint64_t key = uint64_t(m);
  for (int j = 0; j < m; ++j) {
    uint64_t fm = 0;
    for (int i = 0; i < 5; ++i) fm |= 1ull << P.u[j].fcol[i];
    key |= fm << (4 + 12 * j);
  }
  // the store cost depends on which tile bits store to index bits 0..3
  for (int s = 0; s < 4; ++s) {
    uint64_t tb = 15;
    for (int b = 0; b < kTcTileBits; ++b)
      if (P.qt_out[b] == s) tb = uint64_t(b);
    key |= tb << (40 + 4 * s);
  }
  auto apply = [&](const LayoutCfg& best) {
    for (int j = 0; j < m; ++j) {
      for (int i = 0; i < 5; ++i) P.u[j].fcol[i] = best.fcol[j][i];
      for (int i = 0; i < 7; ++i) P.u[j].frow[i] = best.frow[j][i];
    }
    for (int b = 0; b < 11; ++b) P.lt[b] = best.lt[b];
  };
  {
    std::lock_guard<std::mutex> lk(g_layout_mu);
    auto it = g_layout_cache.find(key);
    if (it != g_layout_cache.end()) {
      apply(it->second);
      return;
    }
  }
  LayoutCfg cur;
  for (int j = 0; j < m; ++j) {
    for (int i = 0; i < 5; ++i) cur.fcol[j][i] = P.u[j].fcol[i];
    uint32_t fm = 0;
    for (int i = 0; i < 5; ++i) fm |= 1u << cur.fcol[j][i];
    int r = 0;
    for (int b = 0; b < kTcTileBits; ++b)
      if (!((fm >> b) & 1u)) cur.frow[j][r++] = b;
  }
  for (int b = 0; b < 11; ++b) cur.lt[b] = b + 1;
  uint64_t rng = 0x9E3779B97F4A7C15ull ^ (key * 0xD1B54A32D192ED03ull);  // a function of the cache key only
  auto rnd = [&](int k) {
    rng ^= rng << 13;
    rng ^= rng >> 7;
    rng ^= rng << 17;
    return int(rng % uint64_t(k));
  };
  auto descend = [&](LayoutCfg& c) {
    int cc = layout_cost(c, m, P.qt_out);
    for (int iter = 0; iter < 64; ++iter) {
      int best = cc;
      LayoutCfg bc = c;
      auto consider = [&](const LayoutCfg& t) {
        const int v = layout_cost(t, m, P.qt_out);
        if (v < best) {
          best = v;
          bc = t;
        }
      };
      for (int j = 0; j < m; ++j) {
        for (int a = 0; a < 5; ++a)
          for (int b = a + 1; b < 5; ++b) {
            LayoutCfg t = c;
            std::swap(t.fcol[j][a], t.fcol[j][b]);
            consider(t);
          }
        for (int a = 0; a < 5; ++a)  // rows 5, 6 carry no cost: swaps among them are skipped
          for (int b = a + 1; b < 7; ++b) {
            LayoutCfg t = c;
            std::swap(t.frow[j][a], t.frow[j][b]);
            consider(t);
          }
      }
      for (int a = 3; a < 5; ++a)  // loader lane bits 3, 4 (lane bits 0..2 stay on qubits 1..3)
        for (int b = 3; b < 11; ++b) {
          if (a == b) continue;
          LayoutCfg t = c;
          std::swap(t.lt[a], t.lt[b]);
          consider(t);
        }
      if (best >= cc) break;
      c = bc;
      cc = best;
    }
    return cc;
  };
  LayoutCfg best = cur;
  int bestc = descend(best);
  // lower bound: conflict-free stores (the loader's stores move 256
  // wavefronts per tile, as does each epilogue into a next operand) and fully
  // used HBM sectors
  const int bound = 256 * m;
  for (int restart = 0; restart < 40 && bestc > bound; ++restart) {
    LayoutCfg t = cur;
    for (int j = 0; j < m; ++j) {
      for (int i = 4; i > 0; --i) std::swap(t.fcol[j][i], t.fcol[j][rnd(i + 1)]);
      for (int i = 6; i > 0; --i) std::swap(t.frow[j][i], t.frow[j][rnd(i + 1)]);
    }
    for (int i = 10; i > 3; --i) std::swap(t.lt[i], t.lt[3 + rnd(i - 2)]);
    const int v = descend(t);
    if (v < bestc) {
      bestc = v;
      best = t;
    }
  }
  apply(best);
  std::lock_guard<std::mutex> lk(g_layout_mu);
  if (g_layout_cache.size() >= 65536) g_layout_cache.clear();
  g_layout_cache.emplace(key, best);
}

}  // namespace

uint16_t tc_half_bits(float x) {
  uint32_t f;
  std::memcpy(&f, &x, 4);
  const uint32_t sign = (f >> 16) & 0x8000u;
  const uint32_t absf = f & 0x7FFFFFFFu;
  if (absf >= 0x7F800000u) return uint16_t(sign | 0x7C00u | (absf > 0x7F800000u ? 0x200u : 0u));  // inf / nan
  if (absf >= 0x477FF000u) return uint16_t(sign | 0x7C00u);  // rounds past 65504: overflow to inf
  if (absf < 0x38800000u) {
    // subnormal half (|x| < 2^-14): value = m * 2^-24, round to nearest even
    if (absf < 0x33000000u) return uint16_t(sign);  // below half of the smallest subnormal
    const uint32_t e = absf >> 23;
    const uint32_t mant = (absf & 0x7FFFFFu) | 0x800000u;
    const uint32_t shift = 126u - e;  // 14 + (127 - e) - 1 - 10 + 24 - 23 ...: bits dropped
    const uint32_t q = mant >> shift, rem = mant & ((1u << shift) - 1u), half = 1u << (shift - 1u);
    const uint32_t r = q + ((rem > half || (rem == half && (q & 1u))) ? 1u : 0u);
    return uint16_t(sign | r);
  }
  // normal: re-bias the exponent, round the mantissa to 10 bits (nearest even)
  const uint32_t rem = absf & 0x1FFFu, base = (absf - 0x38000000u) >> 13;
  const uint32_t r = base + ((rem > 0x1000u || (rem == 0x1000u && (base & 1u))) ? 1u : 0u);
  return uint16_t(sign | r);
}

float tc_half_value(uint16_t h) {
  const uint32_t sign = uint32_t(h & 0x8000u) << 16, e = (h >> 10) & 0x1Fu, mant = h & 0x3FFu;
  uint32_t f;
  if (e == 0) {
    const float v = float(mant) * 5.9604644775390625e-8f;  // 2^-24
    return (h & 0x8000u) ? -v : v;
  }
  if (e == 31) f = sign | 0x7F800000u | (mant << 13);
  else f = sign | ((e + 112u) << 23) | (mant << 13);
  float out;
  std::memcpy(&out, &f, 4);
  return out;
}

float tc_state_scale(int n) {
  const int e = std::min(std::max(n / 2 - 2, 0), 12);
  return float(1u << e);
}

bool build_tc_plan(const std::vector<Op>& ops, int n, TcPlan* out, std::string* err, bool finish) {
  out->n = n;
  out->state_scale = tc_state_scale(n);
  out->passes.clear();
  out->bmats.clear();
  out->unitaries.clear();
  out->lq.clear();
  out->stats = PlanStats{};
  if (n < kTcMinQubits || n > kMaxQubits) {
    if (err) *err = "the tensor-core pass mode needs 12 <= n <= 34 qubits";
    return false;
  }
  std::vector<std::vector<int>> cluster_ops;  // ops of each unitary, in pass order
  std::vector<int> remaining(ops.size());
  for (size_t i = 0; i < ops.size(); ++i) remaining[i] = int(i);
  // qubit placement: at[p] = qubit on state index bit p, pos[q] = index bit of
  // qubit q.  Invariant: every displaced qubit is one of a swap pair (l, X),
  // l < 4 <= X: qubit X on bit l and qubit l on bit X.
  std::vector<int> at(static_cast<size_t>(n)), pos(static_cast<size_t>(n));
  for (int q = 0; q < n; ++q) at[size_t(q)] = pos[size_t(q)] = q;
  auto low_qubits = [&]() {
    uint64_t m_ = 0;
    for (int l = 0; l < kTcLowBits; ++l) m_ |= 1ull << at[size_t(l)];
    return m_;
  };
  auto placed_home = [&]() {
    for (int l = 0; l < kTcLowBits; ++l)
      if (at[size_t(l)] != l) return false;
    return true;
  };
  while (!remaining.empty() || !placed_home()) {
    // ---- ops of the pass (the qubits on bits 0..3 are always in the tile) ----
    uint64_t Q = low_qubits(), blocked = 0;
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
    if (clusters.empty()) clusters.emplace_back(0, std::vector<int>());  // a placement-only pass: identity
    // ---- the qubits the next pass wants on bits 0..3: the first qubits of
    // the ops still to come (none left: the displaced low qubits, to go home) ----
    std::vector<int> want;
    {
      uint64_t seen = 0;
      for (int idx : rest) {
        uint64_t qm = ops[size_t(idx)].qubit_mask() & ~seen;
        while (qm && want.size() < size_t(kTcTileBits)) {
          const int q = __builtin_ctzll(qm);
          qm &= qm - 1;
          seen |= 1ull << q;
          want.push_back(q);
        }
        if (want.size() >= size_t(kTcTileBits)) break;
      }
      if (rest.empty())
        for (int l = 0; l < kTcLowBits; ++l)
          if (at[size_t(l)] != l) want.push_back(l);
    }
    // fill the tile to 12 qubits: wanted qubits first (they can then be
    // placed on bits 0..3 by this pass's stores), then the lowest unused
    for (int q : want)
      if (popc(Q) < kTcTileBits) Q |= 1ull << q;
    for (int q = 0; q < n && popc(Q) < kTcTileBits; ++q) Q |= 1ull << q;
    // ---- placement after the pass: wanted qubits onto bits 0..3 by swaps
    // inside the tile (the tile's index bits are pos[Q]) ----
    std::vector<int> at_new = at, pos_new = pos;
    {
      auto in_tile = [&](int q) { return ((Q >> q) & 1ull) != 0; };
      // at most kTcLowBits wanted qubits that are in the tile, in order of need
      std::vector<int> cand;
      for (int q : want)
        if (in_tile(q) && cand.size() < size_t(kTcLowBits)) cand.push_back(q);
      auto is_cand = [&](int q) { return std::find(cand.begin(), cand.end(), q) != cand.end(); };
      bool fixed[kTcLowBits] = {};
      for (int l = 0; l < kTcLowBits; ++l)
        if (is_cand(at_new[size_t(l)])) fixed[l] = true;  // already where it is wanted
      for (int y : cand) {
        if (pos_new[size_t(y)] < kTcLowBits) continue;  // already on bits 0..3
        if (y < kTcLowBits) {
          // a low qubit displaced to bit X: swap it home if bit y is free to change
          if (fixed[y]) continue;
          const int x = at_new[size_t(y)];  // the qubit on bit y, whose home bit holds y
          if (!in_tile(x)) continue;
          at_new[size_t(y)] = y;
          pos_new[size_t(y)] = y;
          at_new[size_t(x)] = x;
          pos_new[size_t(x)] = x;
          fixed[y] = true;
          continue;
        }
        // y >= 5 sits on its own bit y (the invariant): pick a low bit l to swap with
        int best = -1;
        for (int l = 0; l < kTcLowBits && best < 0; ++l)
          if (!fixed[l] && at_new[size_t(l)] == l) best = l;  // bit l holds qubit l: a fresh pair
        for (int l = 0; l < kTcLowBits && best < 0; ++l)
          if (!fixed[l] && at_new[size_t(l)] != l && in_tile(l)) best = l;  // end the pair on bit l first
        if (best < 0) continue;
        const int l = best;
        if (at_new[size_t(l)] != l) {
          const int x = at_new[size_t(l)];  // qubit x on bit l, qubit l on bit x: x goes home
          at_new[size_t(x)] = x;
          pos_new[size_t(x)] = x;
          at_new[size_t(l)] = l;
          pos_new[size_t(l)] = l;
        }
        at_new[size_t(l)] = y;
        pos_new[size_t(y)] = l;
        at_new[size_t(y)] = l;
        pos_new[size_t(l)] = y;
        fixed[l] = true;
      }
    }

    TcPassRec P;
    std::memset(&P, 0, sizeof(P));
    P.m = int(clusters.size());
    for (int s = 0; s < 3; ++s) P.sw_lane[s] = -1;
    std::array<int32_t, kTcTileBits> lq{};
    {
      // tile bits in the order of their index bits when loaded (bits 0..3
      // first: the 128-byte runs); the stores use the new placement
      int b = 0;
      for (int p = 0; p < n; ++p)
        if ((Q >> at[size_t(p)]) & 1ull) {
          lq[size_t(b)] = at[size_t(p)];
          P.qt[b] = p;
          P.qt_out[b] = pos_new[size_t(at[size_t(p)])];
          ++b;
        }
      int o = 0;
      for (int p = 0; p < n; ++p)
        if (!((Q >> at[size_t(p)]) & 1ull)) P.qout[o++] = p;
      P.n_out = o;
    }
    for (int j = 0; j < P.m; ++j) {
      uint64_t F = clusters[size_t(j)].first;
      // pad to exactly 5 qubits with the lowest unused tile qubits
      for (int b = 0; b < kTcTileBits && popc(F) < 5; ++b) F |= 1ull << lq[size_t(b)];
      int i = 0;
      for (int b = 0; b < kTcTileBits; ++b)
        if ((F >> lq[size_t(b)]) & 1ull) P.u[j].fcol[i++] = b;
    }
    out->passes.push_back(P);
    out->lq.push_back(lq);
    for (auto& cl : clusters) cluster_ops.push_back(std::move(cl.second));
    out->stats.stages += uint64_t(P.m);
    remaining.swap(rest);
    at.swap(at_new);
    pos.swap(pos_new);
  }
  if (!finish) {
    out->stats.passes = out->passes.size();
    out->stats.ops = ops.size();
    out->stats.upload_bytes = out->passes.size() * sizeof(TcPassRec) + out->stats.stages * kTcBmatHalves * sizeof(uint16_t);
    return true;
  }
  // ---- per pass (independent, on host threads): layouts, offset tables,
  // unitaries and their split real embeddings ----
  const size_t np = out->passes.size();
  std::vector<size_t> first_u(np + 1, 0);
  for (size_t i = 0; i < np; ++i) first_u[i + 1] = first_u[i] + size_t(out->passes[i].m);
  out->unitaries.assign(first_u[np], {});
  out->bmats.assign(first_u[np] * kTcBmatHalves, uint16_t(0));
  auto finish_pass = [&](size_t pi) {
    TcPassRec& P = out->passes[pi];
    choose_layouts(P);
    for (int j = 0; j < P.m; ++j) layout_offsets(P.u[j].frow, P.u[j].fcol, P.u[j].boff);
    if (!tc_raw_offsets(P.u[0].frow, P.lt, P.roff)) {
      // (the layout cost rules this out; kept valid in any case) a loader bit
      // on row bits 2..6 of unitary 0 becomes the split's half bit: lt[0..2]
      // hold at most three of those five tile bits, so lt[3..9] holds one
      auto on_rows = [&](int tb) {
        for (int i = 2; i < 7; ++i)
          if (P.u[0].frow[i] == tb) return true;
        return false;
      };
      for (int b = 9; b >= 3; --b)
        if (on_rows(P.lt[b])) {
          std::swap(P.lt[b], P.lt[10]);
          break;
        }
      tc_raw_offsets(P.u[0].frow, P.lt, P.roff);
    }
    lane_swaps(P.u[P.m - 1].frow, P.u[P.m - 1].fcol, P.qt_out, P.sw_lane);
    int32_t st_row[7], st_col[5];
    tc_store_bits(P, st_row, st_col);
    for (int j = 0; j < P.m; ++j) {
      TcUnitaryRec& U = P.u[j];
      for (uint32_t c = 0; c < 32; ++c) {
        uint32_t x = 0;
        uint64_t g = 0;
        for (int i = 0; i < 5; ++i)
          if ((c >> i) & 1u) {
            if (j + 1 < P.m) x ^= P.u[j + 1].boff[U.fcol[i]];
            g |= 1ull << (j + 1 == P.m ? st_col[i] : P.qt_out[U.fcol[i]]);
          }
        U.xnext[c] = x;
        U.gcol[c] = g;
      }
    }
    for (int j = 0; j < P.m; ++j) {
      const size_t ui = first_u[pi] + size_t(j);
      int q[5];
      for (int i = 0; i < 5; ++i) q[i] = out->lq[pi][size_t(P.u[j].fcol[i])];
      std::vector<cplx> u(32 * 32, cplx(0, 0));
      for (int c = 0; c < 32; ++c) {
        cplx col[32];
        for (int r = 0; r < 32; ++r) col[r] = (r == c) ? cplx(1, 0) : cplx(0, 0);
        for (int idx : cluster_ops[ui]) fusion_apply_local(ops[size_t(idx)], q, col);
        for (int r = 0; r < 32; ++r) u[size_t(r * 32 + c)] = col[r];
      }
      uint16_t* B = out->bmats.data() + ui * kTcBmatHalves;
      for (int co = 0; co < 32; ++co)
        for (int ci = 0; ci < 32; ++ci) {
          const cplx v = double(kTcUScale) * u[size_t(co * 32 + ci)];
          const double e[2][2] = {{v.real(), -v.imag()}, {v.imag(), v.real()}};
          for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
              const int nrow = 2 * co + a, k = 2 * ci + b;
              const uint16_t hi = tc_half_bits(float(e[a][b]));
              const uint16_t lo = tc_half_bits(float(e[a][b] - double(tc_half_value(hi))));
              B[nrow * 64 + k] = hi;
              B[(64 + nrow) * 64 + k] = lo;
            }
        }
      out->unitaries[ui] = std::move(u);
    }
  };
  {
    const size_t hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t nt = std::min(hw, std::max<size_t>(1, np / 4));
    std::vector<std::thread> th;
    auto work = [&](size_t t) {
      for (size_t pi = t; pi < np; pi += nt) finish_pass(pi);
    };
    for (size_t t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
  }
  out->stats.passes = out->passes.size();
  out->stats.ops = ops.size();
  out->stats.upload_bytes = out->passes.size() * sizeof(TcPassRec) + out->bmats.size() * sizeof(uint16_t);
  return true;
}

}  // namespace nqpu
