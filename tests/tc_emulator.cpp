// Test infrastructure: a CPU emulation of the tensor-core pass kernel
// (nqpu_b200/csrc/tcpass.cu).  It executes the planner's pass records with the
// kernel's index arithmetic — the loader's per-thread / per-step address and
// operand-offset parts, the 128-byte-swizzled K-major FP16 operand images, the
// B operand copy, the contraction D = A B^T over those images, the epilogue's
// row / column offset tables into the next operand layout or HBM, the state
// and unitary scale factors, and the 8- and 16-byte pairing conditions — in
// FP64, optionally with the kernel's FP16 hi/lo split.  Every operand slot and
// every amplitude must be written exactly once per tile, which checks that
// each layout is a bijection.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "planner.h"
#include "tcpass.h"

using namespace nqpu;

namespace {

double half_round(double x) { return double(tc_half_value(tc_half_bits(float(x)))); }

// One FP16 operand plane pair: 8192 half slots each, indexed by byte offset / 2.
struct Operand {
  std::vector<double> hi, lo;
  std::vector<int> written;
  void clear() {
    hi.assign(8192, 0.0);
    lo.assign(8192, 0.0);
    written.assign(8192, 0);
  }
  // store the (re, im) half pair at byte offset o (4-byte aligned), as the
  // kernel's split does: hi = half(x), lo = half(x - hi), x an fp32 value
  bool put(uint32_t o, double re, double im, bool split) {
    if (o % 4 != 0 || o + 4 > 16384) return false;
    const uint32_t s = o / 2;
    if (written[s] || written[s + 1]) return false;
    written[s] = written[s + 1] = 1;
    const double v[2] = {re, im};
    for (int i = 0; i < 2; ++i) {
      if (split) {
        const float x = float(v[i]);
        const double h = half_round(x);
        hi[s + i] = h;
        lo[s + i] = half_round(double(x) - h);
      } else {
        hi[s + i] = v[i];
        lo[s + i] = 0.0;
      }
    }
    return true;
  }
};

}  // namespace

extern "C" uint16_t emu_half_bits(float x) { return tc_half_bits(x); }

// Returns the number of passes (>= 0) or a negative error code:
// -1 plan failed, -2 operand slot written twice / misaligned, -3 amplitude
// written twice or not at all, -4 a pairing condition does not hold,
// -5 the loader's bit map is not a permutation with tile bits 1..3 first,
// -6 the last epilogue's lane exchanges are not distinct lane bits 0..4,
// -7 the raw landing offsets are not a bijection onto 16-byte slots, or a
// half of the two-phase split overwrites a raw chunk not yet read.
extern "C" int emu_tc_run(int n, const double* flat, int ngates, double* state, int split, int64_t* stats) {
  std::vector<GateRec> gates(static_cast<size_t>(ngates));
  for (int i = 0; i < ngates; ++i) {
    const double* g = flat + size_t(i) * 40;
    GateRec& r = gates[size_t(i)];
    r.code = uint8_t(g[0]);
    r.nq = uint8_t(gate_arity(r.code));
    for (int j = 0; j < 3; ++j) r.q[j] = int(g[1 + j]);
    for (int j = 0; j < 4; ++j) r.p[j] = g[4 + j];
    for (int j = 0; j < 16; ++j) r.m[j] = cplx(g[8 + 2 * j], g[9 + 2 * j]);
  }
  TcPlan plan;
  std::string err;
  if (!build_tc_plan(lower_circuit(gates), n, &plan, &err)) return -1;
  const size_t dim = size_t(1) << n;
  const double sc = plan.state_scale, uinv = 1.0 / double(kTcUScale);
  std::vector<double> st(state, state + 2 * dim);
  const uint64_t n_tiles = 1ull << (n - kTcTileBits);
  size_t boff_base = 0;
  int64_t unitaries = 0;
  const int nthr = 1 << kTcLoadThreadBits, nstep = 1 << kTcLoadStepBits;
  for (const TcPassRec& P : plan.passes) {
    const int m = P.m;
    unitaries += m;
    // B operands as the kernel's shared-memory images (FP64 mode: the exact
    // real embedding of 16 U in rows 0..63 and zeros in rows 64..127, so the
    // algebra is checked exactly)
    std::vector<std::vector<double>> bimg(static_cast<size_t>(m), std::vector<double>(8192, 0.0));
    for (int j = 0; j < m; ++j) {
      const uint16_t* B = plan.bmats.data() + boff_base + size_t(j) * kTcBmatHalves;
      const std::vector<cplx>& U = plan.unitaries[size_t(unitaries - m + j)];
      for (uint32_t nrow = 0; nrow < 128; ++nrow)
        for (uint32_t k = 0; k < 64; ++k) {
          double v = tc_half_value(B[nrow * 64 + k]);
          if (!split) {
            const cplx u = nrow < 64 ? double(kTcUScale) * U[(nrow / 2) * 32 + k / 2] : cplx(0, 0);
            const double e[2][2] = {{u.real(), -u.imag()}, {u.imag(), u.real()}};
            v = nrow < 64 ? e[nrow & 1][k & 1] : 0.0;
          }
          bimg[size_t(j)][tc_sw128_off(nrow, k) / 2] = v;
        }
    }
    boff_base += size_t(m) * kTcBmatHalves;
    // loader tables (kernel: T->sol / T->sgl and the per-thread pol / pgl):
    // thread bit b -> tile bit lt[b], step bit s -> tile bit lt[kTcLoadThreadBits + s],
    // tile bit 0 = the pair inside a 16-byte load
    std::vector<uint32_t> sol(size_t(nstep), 0);
    std::vector<uint64_t> sgl(size_t(nstep), 0);
    for (int i = 0; i < nstep; ++i)
      for (int s = 0; s < kTcLoadStepBits; ++s)
        if ((i >> s) & 1) {
          sol[size_t(i)] ^= P.u[0].boff[P.lt[kTcLoadThreadBits + s]];
          sgl[size_t(i)] |= 1ull << P.qt[P.lt[kTcLoadThreadBits + s]];
        }
    {
      uint32_t seen = 1u;  // the loader map must be a permutation of tile bits 1..11
      for (int b = 0; b < 11; ++b) {
        if (P.lt[b] < 1 || P.lt[b] > 11 || ((seen >> P.lt[b]) & 1u)) return -5;
        seen |= 1u << P.lt[b];
      }
      if (P.lt[0] != 1 || P.lt[1] != 2 || P.lt[2] != 3) return -5;
    }
    // last epilogue: lane bit sw_lane[s] trades places with column bit 1 + s
    // (a warp shuffle in the kernel); the store-side index bits of the row
    // and column bits follow the exchange
    int32_t st_row[7], st_col[5];
    tc_store_bits(P, st_row, st_col);
    {
      uint32_t seen = 0;
      for (int s = 0; s < 3; ++s) {
        const int l = P.sw_lane[s];
        if (l < -1 || l > 4 || (l >= 0 && ((seen >> l) & 1u))) return -6;
        if (l >= 0) seen |= 1u << l;
      }
    }
    // the kernel forms the epilogue offsets from one entry per column bit:
    // xnext and gcol must be linear (XOR of the next layout's offsets, sum of
    // the qubits' amplitude strides) in the bits of the column index
    for (int j = 0; j < m; ++j)
      for (uint32_t c = 0; c < 32; ++c) {
        uint32_t x = 0;
        uint64_t g = 0;
        for (int i = 0; i < 5; ++i)
          if ((c >> i) & 1u) {
            if (j + 1 < m) x ^= P.u[j + 1].boff[P.u[j].fcol[i]];
            g += 1ull << (j + 1 == m ? st_col[i] : P.qt_out[P.u[j].fcol[i]]);
          }
        if ((j + 1 < m && P.u[j].xnext[c] != x) || (j + 1 == m && P.u[j].gcol[c] != g)) return -4;
      }
    const uint32_t boff_h = P.u[0].boff[0];
    const bool load_pair = boff_h == 4u;  // tile bit 0 is column bit 0 of unitary 0
    {
      // raw landing (kernel: raw_t ^ the step bits' T->rsb): chunk (thread gt,
      // step i) lands at a 16-byte slot of the 32 KB operand buffer; the split
      // reads the chunks of load-step bit 3 = 0, meets, writes their hi / lo
      // outputs, then the same for bit 3 = 1.  No write may hit a slot whose
      // raw chunk is still unread.
      std::vector<int> owner(2048, -1);
      std::vector<char> done(size_t(nthr * nstep), 0);
      auto chunk_raw = [&](int gt, int i) {
        uint32_t r = 0;
        for (int b = 0; b < kTcLoadThreadBits; ++b)
          if ((gt >> b) & 1) r ^= P.roff[P.lt[b]];
        for (int b = 0; b < kTcLoadStepBits; ++b)
          if ((i >> b) & 1) r ^= P.roff[P.lt[kTcLoadThreadBits + b]];
        return r;
      };
      for (int gt = 0; gt < nthr; ++gt)
        for (int i = 0; i < nstep; ++i) {
          const uint32_t r = chunk_raw(gt, i);
          if ((r & 15u) || r >= 32768u || owner[r >> 4] >= 0) return -7;
          owner[r >> 4] = gt * nstep + i;
        }
      for (int h = 0; h < 2; ++h) {
        for (int gt = 0; gt < nthr; ++gt)
          for (int i = 0; i < nstep; ++i)
            if ((i >> 3) == h) done[size_t(gt * nstep + i)] = 1;
        for (int gt = 0; gt < nthr; ++gt) {
          uint32_t pol = 0;
          for (int b = 0; b < kTcLoadThreadBits; ++b)
            if ((gt >> b) & 1) pol ^= P.u[0].boff[P.lt[b]];
          for (int i = 0; i < nstep; ++i) {
            if ((i >> 3) != h) continue;
            const uint32_t o = pol ^ sol[size_t(i)];
            for (uint32_t u : {o, o ^ boff_h, o + 16384u, (o ^ boff_h) + 16384u}) {
              const int w = owner[u >> 4];
              if (w >= 0 && !done[size_t(w)]) return -7;
            }
          }
        }
      }
    }
    const bool store16 = P.qt_out[P.u[m - 1].fcol[0]] == 0;
    std::vector<int> amp_written(dim, 0);
    for (uint64_t tile = 0; tile < n_tiles; ++tile) {
      uint64_t tb = 0;
      for (int j = 0; j < P.n_out; ++j)
        if ((tile >> j) & 1ull) tb |= 1ull << P.qout[j];
      Operand A;
      A.clear();
      for (int gt = 0; gt < nthr; ++gt) {
        uint32_t pol = 0;
        uint64_t pgl = 0;
        for (int b = 0; b < kTcLoadThreadBits; ++b)
          if ((gt >> b) & 1) {
            pol ^= P.u[0].boff[P.lt[b]];
            pgl |= 1ull << P.qt[P.lt[b]];
          }
        for (int i = 0; i < nstep; ++i) {
          const uint64_t a = tb + pgl + sgl[size_t(i)];  // even: the 16-byte load of amplitudes a, a + 1
          if (a & 1ull) return -3;
          const uint32_t o = pol ^ sol[size_t(i)];
          if (load_pair && ((o & 7u) || (o ^ boff_h) != o + 4)) return -4;
          if (!A.put(o, sc * st[2 * a], sc * st[2 * a + 1], split != 0)) return -2;
          if (!A.put(o ^ boff_h, sc * st[2 * a + 2], sc * st[2 * a + 3], split != 0)) return -2;
        }
      }
      for (int s = 0; s < 8192; ++s)
        if (!A.written[size_t(s)]) return -2;
      for (int j = 0; j < m; ++j) {
        const std::vector<double>& Bi = bimg[size_t(j)];
        // D[r][0:128] = A_hi [B_hi; B_lo]^T ; D[r][0:64] += A_lo B_hi^T
        std::vector<double> D(128 * 128, 0.0);
        for (uint32_t r = 0; r < 128; ++r)
          for (uint32_t nn = 0; nn < 128; ++nn) {
            double acc = 0.0;
            for (uint32_t k = 0; k < 64; ++k) {
              const uint32_t ao = tc_sw128_off(r, k) / 2, bo = tc_sw128_off(nn, k) / 2;
              acc += A.hi[ao] * Bi[bo];
              if (nn < 64) acc += A.lo[ao] * Bi[bo];
            }
            D[r * 128 + nn] = acc;
          }
        const bool last = j + 1 == m;
        Operand N;
        N.clear();
        for (uint32_t r = 0; r < 128; ++r) {
          uint32_t ptn = 0;
          uint64_t pg = 0;
          for (int i = 0; i < 7; ++i)
            if ((r >> i) & 1u) {
              if (!last) ptn ^= P.u[j + 1].boff[P.u[j].frow[i]];
              else pg |= 1ull << st_row[i];
            }
          const bool pair = !last && P.u[j + 1].boff[P.u[j].fcol[0]] == 4u;
          for (uint32_t c = 0; c < 32; ++c) {
            // the thread of row r holds, in its register of column c, the
            // element (rs, cs): after the lane exchanges of the last epilogue,
            // row bit sw_lane[s] comes from c's bit 1 + s and vice versa
            uint32_t rs = r, cs = c;
            if (last)
              for (int s = 0; s < 3; ++s) {
                const int l = P.sw_lane[s];
                if (l < 0) continue;
                const uint32_t rb = (r >> l) & 1u, cb = (c >> (1 + s)) & 1u;
                rs = (rs & ~(1u << l)) | (cb << l);
                cs = (cs & ~(1u << (1 + s))) | (rb << (1 + s));
              }
            double re = (D[rs * 128 + 2 * cs] + D[rs * 128 + 64 + 2 * cs]) * uinv;
            double im = (D[rs * 128 + 2 * cs + 1] + D[rs * 128 + 64 + 2 * cs + 1]) * uinv;
            if (split) {
              re = double(float(re));
              im = double(float(im));
            }
            if (!last) {
              const uint32_t o = ptn ^ P.u[j].xnext[c];
              if (pair && (c & 1u) == 0 && ((o & 7u) || (ptn ^ P.u[j].xnext[c + 1]) != o + 4)) return -4;
              if (!N.put(o, re, im, split != 0)) return -2;
            } else {
              const uint64_t a = tb + pg + P.u[j].gcol[c];
              if (store16 && (c & 1u) == 0 && (a & 1ull)) return -4;
              if (store16 && (c & 1u) == 1 && P.u[j].gcol[c] != P.u[j].gcol[c - 1] + 1) return -4;
              if (a >= dim || amp_written[a]) return -3;
              amp_written[a] = 1;
              st[2 * a] = re / sc;
              st[2 * a + 1] = im / sc;
            }
          }
        }
        if (!last) {
          for (int s = 0; s < 8192; ++s)
            if (!N.written[size_t(s)]) return -2;
          A = N;
        }
      }
    }
    for (size_t a = 0; a < dim; ++a)
      if (!amp_written[a]) return -3;
  }
  std::memcpy(state, st.data(), sizeof(double) * 2 * dim);
  if (stats) {
    stats[0] = int64_t(plan.passes.size());
    stats[1] = unitaries;
    stats[2] = int64_t(plan.stats.upload_bytes);
  }
  return int(plan.passes.size());
}

// Plan only: the 128-byte lines one warp store of each pass's last epilogue
// touches (2^k, k = lane bits storing to index bits >= 4), summed over the
// passes, with (out[0]) and without (out[1]) the lane exchanges, and the
// exchanges made (out[2]).  Returns the number of passes or -1.
extern "C" int emu_tc_store_lines(int n, const double* flat, int ngates, int64_t* out) {
  std::vector<GateRec> gates(static_cast<size_t>(ngates));
  for (int i = 0; i < ngates; ++i) {
    const double* g = flat + size_t(i) * 40;
    GateRec& r = gates[size_t(i)];
    r.code = uint8_t(g[0]);
    r.nq = uint8_t(gate_arity(r.code));
    for (int j = 0; j < 3; ++j) r.q[j] = int(g[1 + j]);
    for (int j = 0; j < 4; ++j) r.p[j] = g[4 + j];
    for (int j = 0; j < 16; ++j) r.m[j] = cplx(g[8 + 2 * j], g[9 + 2 * j]);
  }
  TcPlan plan;
  std::string err;
  if (!build_tc_plan(lower_circuit(gates), n, &plan, &err)) return -1;
  out[0] = out[1] = out[2] = 0;
  for (const TcPassRec& P : plan.passes) {
    int32_t st_row[7], st_col[5];
    tc_store_bits(P, st_row, st_col);
    int k = 0, k0 = 0;
    for (int i = 0; i < 5; ++i) {
      k += st_row[i] >= 4 ? 1 : 0;
      k0 += P.qt_out[P.u[P.m - 1].frow[i]] >= 4 ? 1 : 0;
    }
    out[0] += int64_t(1) << k;
    out[1] += int64_t(1) << k0;
    for (int s = 0; s < 3; ++s) out[2] += P.sw_lane[s] >= 0 ? 1 : 0;
  }
  return int(plan.passes.size());
}

// The raw landing alone (tcpass.h: tc_raw_offsets), over `trials` seeded random
// layouts of unitary 0 (row / column orders) and loader maps: for every valid
// choice (half bit lt[10] on row bits 2..6), the 2048 chunks must land on
// distinct 16-byte slots of the 32 KB buffer, and every chunk of half h must
// land in a slot that only half h's hi / lo outputs fill.  Returns the number
// of valid layouts checked, or -1 on the first violation.
extern "C" int emu_tc_raw_landing(int trials, uint64_t seed) {
  uint64_t s = seed | 1u;
  auto rnd = [&](int k) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return int(s % uint64_t(k));
  };
  int valid = 0;
  for (int t = 0; t < trials; ++t) {
    int perm[12];
    for (int b = 0; b < 12; ++b) perm[b] = b;
    for (int i = 11; i > 0; --i) std::swap(perm[i], perm[rnd(i + 1)]);
    int32_t frow[7], fcol[5];
    for (int i = 0; i < 7; ++i) frow[i] = perm[i];
    for (int i = 0; i < 5; ++i) fcol[i] = perm[7 + i];
    uint32_t boff[12];
    for (int i = 0; i < 7; ++i) boff[frow[i]] = tc_sw128_off(1u << i, 0);
    for (int i = 0; i < 5; ++i) boff[fcol[i]] = tc_sw128_off(0, 2u << i);
    int32_t lt[11] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11};
    for (int i = 10; i > 3; --i) std::swap(lt[i], lt[3 + rnd(i - 2)]);
    uint32_t roff[12];
    if (!tc_raw_offsets(frow, lt, roff)) continue;
    ++valid;
    std::vector<int> owner(2048, -1);
    for (int c = 0; c < 2048; ++c) {  // chunk bits: loader bits 0..10 -> tile bits lt[.]
      uint32_t r = 0;
      for (int k = 0; k < 11; ++k)
        if ((c >> k) & 1) r ^= roff[lt[k]];
      if ((r & 15u) || r >= 32768u || owner[r >> 4] >= 0) return -1;
      owner[r >> 4] = c;
    }
    for (int c = 0; c < 2048; ++c) {
      const int h = (c >> 10) & 1;  // loader bit 10 = load-step bit 3, the half bit
      uint32_t o = 0;               // hi offset of the chunk's first amplitude (tile bit 0 = 0)
      for (int k = 0; k < 11; ++k)
        if ((c >> k) & 1) o ^= boff[lt[k]];
      for (uint32_t u : {o, o ^ boff[0], o + 16384u, (o ^ boff[0]) + 16384u})
        if (((owner[u >> 4] >> 10) & 1) != h) return -1;
    }
  }
  return valid;
}
