// Device code shared by the tiled pass kernel and the batched executor: the
// shared-memory swizzle, register-block op bodies, op dispatch, the stage
// executor and async-copy helpers.  Included by .cu files only.
#pragma once
#include "sv_device.cuh"

namespace nqpu {

constexpr int kTileThreads = 256;
constexpr int kVecPerThread = 16;
// Tile bits above the contiguous low block: k - c <= 8 (c >= 5 for complex64,
// c >= 4 for complex128, k <= 13 / 12), so the high-offset table has <= 256 entries.
constexpr int kHiOffBits = 8;
constexpr int kHiOffEntries = 1 << kHiOffBits;

__device__ __forceinline__ uint32_t swz(uint32_t u) {
  uint32_t w = u >> 3;
  uint32_t f = w ^ (w >> 3) ^ (w >> 6) ^ (w >> 9) ^ (w >> 12);
  return u ^ (f & 7u);
}

template <typename C>
__device__ __forceinline__ C csel(bool p, C a, C b) {
  C r;
  r.x = p ? a.x : b.x;
  r.y = p ? a.y : b.y;
  return r;
}

// ---- register-block op bodies (B, B0, B1, CB, ... are register-bit indices)
// Every amplitude index i below is a compile-time constant after unrolling, so
// the register block stays in registers; runtime register bits are turned into
// template arguments by the dispatch switches.

template <typename Real>
__device__ __forceinline__ void ldc2(const Real* __restrict__ p, typename Tr<Real>::C& a,
                                     typename Tr<Real>::C& b);
template <>
__device__ __forceinline__ void ldc2<float>(const float* __restrict__ p, float2& a, float2& b) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  a = make_float2(v.x, v.y);
  b = make_float2(v.z, v.w);
}
template <>
__device__ __forceinline__ void ldc2<double>(const double* __restrict__ p, double2& a, double2& b) {
  a = __ldg(reinterpret_cast<const double2*>(p));
  b = __ldg(reinterpret_cast<const double2*>(p) + 1);
}

// complex product on a register amplitude: packed FFMA2 form for complex64
template <typename C>
__device__ __forceinline__ C rmul(C m, C x) {
  if constexpr (sizeof(m.x) == 4) return pcmul(pack_coef(m), x);
  else return cmul(m, x);
}

// dense 2x2, no controls
template <typename C, int NA, int B>
__device__ __forceinline__ void rb_u1(C (&a)[NA], C m0, C m1, C m2, C m3) {
  if constexpr (sizeof(m0.x) == 4) {
    const PackedC p0 = pack_coef(m0), p1 = pack_coef(m1), p2 = pack_coef(m2), p3 = pack_coef(m3);
#pragma unroll
    for (int i = 0; i < NA; ++i) {
      if (i & (1 << B)) continue;
      const int j = i | (1 << B);
      const float2 x = a[i], y = a[j];
      const float2 sx = swap_ri(x), sy = swap_ri(y);
      float2 ti = __fmul2_rn(p0.p, x), tj = __fmul2_rn(p2.p, x);
      ti = __ffma2_rn(p0.q, sx, ti);
      tj = __ffma2_rn(p2.q, sx, tj);
      ti = __ffma2_rn(p1.p, y, ti);
      tj = __ffma2_rn(p3.p, y, tj);
      a[i] = __ffma2_rn(p1.q, sy, ti);
      a[j] = __ffma2_rn(p3.q, sy, tj);
    }
  } else {
#pragma unroll
    for (int i = 0; i < NA; ++i) {
      if (i & (1 << B)) continue;
      const int j = i | (1 << B);
      const C x = a[i], y = a[j];
      a[i] = cmac2(m0, x, m1, y);
      a[j] = cmac2(m2, x, m3, y);
    }
  }
}

// dense 2x2 with controls (generic: per-amplitude select)
template <typename C, int NA, int B>
__device__ __forceinline__ void rb_u1_ctrl(C (&a)[NA], C m0, C m1, C m2, C m3, bool tc, uint32_t creg) {
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    if (i & (1 << B)) continue;
    const int j = i | (1 << B);
    const bool cond = tc && ((uint32_t(i) & creg) == creg);
    const C x = a[i], y = a[j];
    a[i] = csel(cond, cmac2(m0, x, m1, y), x);
    a[j] = csel(cond, cmac2(m2, x, m3, y), y);
  }
}

template <typename C, int NA>
__device__ __forceinline__ void rb_x1_generic(C (&a)[NA], int b, bool tc, uint32_t creg) {
#pragma unroll
  for (int i = 0; i < NA; ++i) {
#pragma unroll
    for (int bb = 0; bb < 5; ++bb) {
      if ((1 << bb) >= NA) break;
      if (bb != b) continue;
      if (i & (1 << bb)) continue;
      const int j = i | (1 << bb);
      const bool cond = tc && ((uint32_t(i) & creg) == creg);
      const C x = a[i], y = a[j];
      a[i] = csel(cond, y, x);
      a[j] = csel(cond, x, y);
    }
  }
}

// X on register bit B, controlled by the register bits CM (compile time) and
// by controls outside the registers (tc): per-thread selects (TC_ALWAYS would
// make it a register renaming, which only straight-line code can afford).
template <typename C, int NA, int B, int CM, bool TC_ALWAYS>
__device__ __forceinline__ void rb_x1_fixed(C (&a)[NA], bool tc) {
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    if (i & (1 << B)) continue;
    if ((i & CM) != CM) continue;
    const int j = i | (1 << B);
    const C x = a[i], y = a[j];
    if constexpr (TC_ALWAYS) {
      a[i] = y;
      a[j] = x;
    } else {
      a[i] = csel(tc, y, x);
      a[j] = csel(tc, x, y);
    }
  }
}

template <typename C, int NA, int NRB, int B, bool TC_ALWAYS>
__device__ __forceinline__ void dispatch_x1_ctrl(C (&a)[NA], uint32_t creg, bool tc) {
  switch (creg) {
#define NQ_X1C(V) case (V == 0 ? 0 : (1 << (V - 1))): \
    if constexpr (V == 0 || (V - 1 < NRB && V - 1 != B)) rb_x1_fixed<C, NA, B, (V == 0 ? 0 : (1 << (V - 1))), TC_ALWAYS>(a, tc); break;
    NQ_X1C(0) NQ_X1C(1) NQ_X1C(2) NQ_X1C(3) NQ_X1C(4) NQ_X1C(5)
#undef NQ_X1C
    default: break;
  }
}

// phase m on the register amplitudes whose bits CMASK are all set
template <typename C, int NA, int CMASK>
__device__ __forceinline__ void rb_ph(C (&a)[NA], C m, bool neg) {
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    if ((i & CMASK) != CMASK) continue;
    if (neg) {
      a[i].x = -a[i].x;
      a[i].y = -a[i].y;
    } else {
      a[i] = rmul(m, a[i]);
    }
  }
}

// diag(d0, d1) selected by register bit DB (DB == NA_BITS: the thread-level bit tb)
template <typename C, int NA, int DB, int NRB>
__device__ __forceinline__ void rb_d1(C (&a)[NA], C d0, C d1, uint32_t tb) {
  if constexpr (DB >= NRB) {
    const C d = csel(tb != 0, d1, d0);
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = rmul(d, a[i]);
  } else {
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = rmul((i & (1 << DB)) ? d1 : d0, a[i]);
  }
}

// diag on two bits (register bit or thread-level bit when >= NRB)
template <typename C, int NA, int D0, int D1, int NRB>
__device__ __forceinline__ void rb_d2(C (&a)[NA], const C* m, uint32_t tb0, uint32_t tb1) {
  if constexpr (D0 >= NRB && D1 >= NRB) {
    const C lo = csel(tb0 != 0, m[1], m[0]);
    const C hi = csel(tb0 != 0, m[3], m[2]);
    const C d = csel(tb1 != 0, hi, lo);
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = rmul(d, a[i]);
  } else if constexpr (D0 >= NRB) {
    const C lo = csel(tb0 != 0, m[1], m[0]);
    const C hi = csel(tb0 != 0, m[3], m[2]);
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = rmul((i & (1 << D1)) ? hi : lo, a[i]);
  } else if constexpr (D1 >= NRB) {
    const C lo = csel(tb1 != 0, m[2], m[0]);
    const C hi = csel(tb1 != 0, m[3], m[1]);
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = rmul((i & (1 << D0)) ? hi : lo, a[i]);
  } else {
#pragma unroll
    for (int i = 0; i < NA; ++i) {
      const int k = ((i >> D0) & 1) | (((i >> D1) & 1) << 1);
      a[i] = rmul(m[k], a[i]);
    }
  }
}

// generic diagonal with controls: d selected per amplitude at run time
template <typename C, int NA>
__device__ __forceinline__ void rb_diag_generic(C (&a)[NA], const C* m, int nd, uint32_t dreg0,
                                                uint32_t dreg1, uint32_t tb0, uint32_t tb1, bool tc,
                                                uint32_t creg) {
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    const bool cond = tc && ((uint32_t(i) & creg) == creg);
    const uint32_t b0 = (dreg0 != 0xFF) ? ((uint32_t(i) >> dreg0) & 1u) : tb0;
    const uint32_t b1 = (nd > 1) ? ((dreg1 != 0xFF) ? ((uint32_t(i) >> dreg1) & 1u) : tb1) : 0u;
    const C lo = csel(b0 != 0, m[1], m[0]);
    const C hi = csel(b0 != 0, m[3], m[2]);
    const C d = csel(b1 != 0, hi, lo);
    a[i] = csel(cond, cmul(d, a[i]), a[i]);
  }
}

// dense 4x4 on register bits (B0 = sub-index bit 0, B1 = bit 1); matrix rows
// are read from the op record (L1-resident) per quad to keep registers free.
template <typename Real, typename C, int NA, int B0, int B1>
__device__ __forceinline__ void rb_u2(C (&a)[NA], const Real* __restrict__ mp, bool tc, uint32_t creg) {
  constexpr int M0 = 1 << B0, M1 = 1 << B1;
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    if (i & (M0 | M1)) continue;
    const bool cond = tc && ((uint32_t(i) & creg) == creg);
    const C x0 = a[i], x1 = a[i | M0], x2 = a[i | M1], x3 = a[i | M0 | M1];
    C y[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      C m[4];
      ldc2<Real>(mp + 8 * r, m[0], m[1]);
      ldc2<Real>(mp + 8 * r + 4, m[2], m[3]);
      y[r] = cmac4(m, x0, x1, x2, x3);
    }
    a[i] = csel(cond, y[0], x0);
    a[i | M0] = csel(cond, y[1], x1);
    a[i | M1] = csel(cond, y[2], x2);
    a[i | M0 | M1] = csel(cond, y[3], x3);
  }
}

template <typename C, int NA, int B0, int B1>
__device__ __forceinline__ void rb_sw(C (&a)[NA], bool tc, uint32_t creg) {
  constexpr int M0 = 1 << B0, M1 = 1 << B1;
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    if (i & (M0 | M1)) continue;
    const bool cond = tc && ((uint32_t(i) & creg) == creg);
    const C x1 = a[i | M0], x2 = a[i | M1];
    a[i | M0] = csel(cond, x2, x1);
    a[i | M1] = csel(cond, x1, x2);
  }
}

// ---- dispatch helpers ------------------------------------------------------
#define NQ_REG_CASES(M, ...) M(0, __VA_ARGS__) M(1, __VA_ARGS__) M(2, __VA_ARGS__) M(3, __VA_ARGS__) M(4, __VA_ARGS__)

template <typename C, int NA, int NRB>
__device__ __forceinline__ void dispatch_ph(C (&a)[NA], uint32_t creg, C m, bool neg) {
  switch (creg) {
#define NQ_PHC(V) case V: if constexpr (V < (1 << NRB)) rb_ph<C, NA, V>(a, m, neg); break;
    NQ_PHC(0) NQ_PHC(1) NQ_PHC(2) NQ_PHC(3) NQ_PHC(4) NQ_PHC(5) NQ_PHC(6) NQ_PHC(7)
    NQ_PHC(8) NQ_PHC(9) NQ_PHC(10) NQ_PHC(11) NQ_PHC(12) NQ_PHC(13) NQ_PHC(14) NQ_PHC(15)
    NQ_PHC(16) NQ_PHC(17) NQ_PHC(18) NQ_PHC(19) NQ_PHC(20) NQ_PHC(21) NQ_PHC(22) NQ_PHC(23)
    NQ_PHC(24) NQ_PHC(25) NQ_PHC(26) NQ_PHC(27) NQ_PHC(28) NQ_PHC(29) NQ_PHC(30) NQ_PHC(31)
#undef NQ_PHC
    default: break;
  }
}

template <typename C, int NA, int NRB, int D0>
__device__ __forceinline__ void dispatch_d2_b(C (&a)[NA], int d1, const C* m, uint32_t tb0, uint32_t tb1) {
  switch (d1) {
#define NQ_D2B(V) case V: if constexpr (V <= NRB && (V != D0 || V == NRB)) rb_d2<C, NA, D0, V, NRB>(a, m, tb0, tb1); break;
    NQ_D2B(0) NQ_D2B(1) NQ_D2B(2) NQ_D2B(3) NQ_D2B(4) NQ_D2B(5)
#undef NQ_D2B
    default: break;
  }
}

template <typename Real, typename C, int NA, int NRB, int B0>
__device__ __forceinline__ void dispatch_u2_b(C (&a)[NA], int b1, const Real* mp, bool tc, uint32_t creg) {
  switch (b1) {
#define NQ_U2B(V) case V: if constexpr (V < NRB && V != B0) rb_u2<Real, C, NA, B0, V>(a, mp, tc, creg); break;
    NQ_U2B(0) NQ_U2B(1) NQ_U2B(2) NQ_U2B(3) NQ_U2B(4)
#undef NQ_U2B
    default: break;
  }
}

template <typename C, int NA, int NRB, int B0>
__device__ __forceinline__ void dispatch_sw_b(C (&a)[NA], int b1, bool tc, uint32_t creg) {
  switch (b1) {
#define NQ_SWB(V) case V: if constexpr (V < NRB && V != B0) rb_sw<C, NA, B0, V>(a, tc, creg); break;
    NQ_SWB(0) NQ_SWB(1) NQ_SWB(2) NQ_SWB(3) NQ_SWB(4)
#undef NQ_SWB
    default: break;
  }
}

// Apply ops [ob, oe) of a stage to the thread's register block.
// vbase = virtual index of register amplitude 0 (register bits are zero in it).
template <typename Real, int NA, int NRB, bool kDiagFlat = false>
__device__ __forceinline__ void apply_stage_ops(typename Tr<Real>::C (&a)[NA],
                                                const TileOp<Real>* __restrict__ ops, int ob,
                                                int oe, uint32_t vbase) {
  using C = typename Tr<Real>::C;
  // software pipeline: the next op's header and first four matrix entries are
  // loaded while the current op runs
  uint4 nh = make_uint4(0, 0, 0, 0);
  uint32_t ndv1 = 0;
  C nm[4];
  auto fetch = [&](int o) {
    const TileOp<Real>* op = ops + o;
    nh = __ldg(reinterpret_cast<const uint4*>(op));
    ndv1 = __ldg(reinterpret_cast<const uint32_t*>(op) + 4);
    ldc2<Real>(op->m, nm[0], nm[1]);
    ldc2<Real>(op->m + 4, nm[2], nm[3]);
  };
  if (ob < oe) fetch(ob);
  for (int o = ob; o < oe; ++o) {
    const TileOp<Real>* op = ops + o;
    const uint4 h0 = nh;
    const uint32_t dv1 = ndv1;
    const C pm0 = nm[0], pm1 = nm[1], pm2 = nm[2], pm3 = nm[3];
    if (o + 1 < oe) fetch(o + 1);
    const uint32_t kind = h0.x & 0xFF;
    const uint32_t rb0 = (h0.x >> 8) & 0xFF;
    const uint32_t rb1 = (h0.x >> 16) & 0xFF;
    const uint32_t creg = (h0.x >> 24) & 0xFF;
    const uint32_t dreg0 = h0.y & 0xFF;
    const uint32_t dreg1 = (h0.y >> 8) & 0xFF;
    const uint32_t cnr = h0.z;
    const uint32_t dv0 = h0.w;
    const bool tc = (vbase & cnr) == cnr;
    const Real* mp = op->m;
    // the common cases (dense 1q gate, X / CNOT with at most one register
    // control) through one flat switch on a code the planner precomputed
    const uint32_t fast = (h0.y >> 16) & 0xFF;
    if (fast != 0) {
      switch (fast) {
#define NQ_FU1(B, _) case 1 + B: if constexpr (B < NRB) { if (tc) rb_u1<C, NA, B>(a, pm0, pm1, pm2, pm3); } break;
        NQ_REG_CASES(NQ_FU1, 0)
#undef NQ_FU1
#define NQ_FX1V(B, V) case 8 + 8 * B + V: \
        if constexpr (B < NRB && (V == 0 || (V - 1 < NRB && V - 1 != B))) \
          rb_x1_fixed<C, NA, B, (V == 0 ? 0 : (1 << (V - 1))), false>(a, tc); \
        break;
#define NQ_FX1(B, _) NQ_FX1V(B, 0) NQ_FX1V(B, 1) NQ_FX1V(B, 2) NQ_FX1V(B, 3) NQ_FX1V(B, 4) NQ_FX1V(B, 5)
        NQ_REG_CASES(NQ_FX1, 0)
#undef NQ_FX1
#undef NQ_FX1V
        default: break;
      }
      continue;
    }
    // the batch executor's variant also takes the diagonal shapes through a
    // flat switch (TileOp::fast2); measured +1 % there, while the tiled pass
    // kernel ran QFT passes 1 % slower with it
    if constexpr (kDiagFlat) {
      const uint32_t fast2 = (h0.y >> 24) & 0xFF;
      if (fast2 != 0) {
        switch (fast2) {
#define NQ_FD1(B) case 48 + B: \
          if constexpr (B <= NRB) rb_d1<C, NA, B, NRB>(a, pm0, pm1, (vbase & dv0) ? 1u : 0u); \
          break;
          NQ_FD1(0) NQ_FD1(1) NQ_FD1(2) NQ_FD1(3) NQ_FD1(4) NQ_FD1(5)
#undef NQ_FD1
#define NQ_FPH(V) case 128 + V: \
          if constexpr (V < (1 << NRB)) { \
            if (tc) rb_ph<C, NA, V>(a, pm0, (pm0.x == Real(-1)) && (pm0.y == Real(0))); \
          } \
          break;
          NQ_FPH(0) NQ_FPH(1) NQ_FPH(2) NQ_FPH(3) NQ_FPH(4) NQ_FPH(5) NQ_FPH(6) NQ_FPH(7)
          NQ_FPH(8) NQ_FPH(9) NQ_FPH(10) NQ_FPH(11) NQ_FPH(12) NQ_FPH(13) NQ_FPH(14) NQ_FPH(15)
          NQ_FPH(16) NQ_FPH(17) NQ_FPH(18) NQ_FPH(19) NQ_FPH(20) NQ_FPH(21) NQ_FPH(22) NQ_FPH(23)
          NQ_FPH(24) NQ_FPH(25) NQ_FPH(26) NQ_FPH(27) NQ_FPH(28) NQ_FPH(29) NQ_FPH(30) NQ_FPH(31)
#undef NQ_FPH
#define NQ_FD2V(D0, D1) case 160 + 8 * D0 + D1: \
          if constexpr (D0 <= NRB && D1 <= NRB && (D0 != D1 || D0 == NRB)) { \
            const C m[4] = {pm0, pm1, pm2, pm3}; \
            rb_d2<C, NA, D0, D1, NRB>(a, m, (vbase & dv0) ? 1u : 0u, (vbase & dv1) ? 1u : 0u); \
          } \
          break;
#define NQ_FD2(D0) NQ_FD2V(D0, 0) NQ_FD2V(D0, 1) NQ_FD2V(D0, 2) NQ_FD2V(D0, 3) NQ_FD2V(D0, 4) NQ_FD2V(D0, 5)
          NQ_FD2(0) NQ_FD2(1) NQ_FD2(2) NQ_FD2(3) NQ_FD2(4) NQ_FD2(5)
#undef NQ_FD2
#undef NQ_FD2V
          default: break;
        }
        continue;
      }
    }
    switch (kind) {
      case OP_U1: {
        const C m0 = pm0, m1 = pm1, m2 = pm2, m3 = pm3;
        if (creg == 0) {
          if (!tc) break;
          switch (rb0) {
#define NQ_U1(B, _) case B: if constexpr (B < NRB) rb_u1<C, NA, B>(a, m0, m1, m2, m3); break;
            NQ_REG_CASES(NQ_U1, 0)
#undef NQ_U1
            default: break;
          }
        } else {
          switch (rb0) {
#define NQ_U1C(B, _) case B: if constexpr (B < NRB) rb_u1_ctrl<C, NA, B>(a, m0, m1, m2, m3, tc, creg); break;
            NQ_REG_CASES(NQ_U1C, 0)
#undef NQ_U1C
            default: break;
          }
        }
        break;
      }
      case OP_X1: {
        // X / CNOT kept in registers because later ops of the stage act on
        // its qubits (the others are deferred into the write-back map).  At
        // most one register control: a fixed register permutation; more
        // (Toffoli): generic per-amplitude selects.
        if (creg & (creg - 1)) {
          rb_x1_generic<C, NA>(a, int(rb0), tc, creg);
          break;
        }
        // selects even when tc is always true: a compile-time register
        // permutation here would make the allocator shuffle (and spill) the
        // register block on every other op's path
        switch (rb0) {
#define NQ_X1(B, _) case B: \
          if constexpr (B < NRB) dispatch_x1_ctrl<C, NA, NRB, B, false>(a, creg, tc); \
          break;
          NQ_REG_CASES(NQ_X1, 0)
#undef NQ_X1
          default: break;
        }
        break;
      }
      case OP_PH: {
        if (!tc) break;
        const C m0 = pm0;
        const bool neg = (m0.x == Real(-1)) && (m0.y == Real(0));
        dispatch_ph<C, NA, NRB>(a, creg, m0, neg);
        break;
      }
      case OP_D1: {
        C m[4];
        m[0] = pm0;
        m[1] = pm1;
        const uint32_t tb = (vbase & dv0) ? 1u : 0u;
        if (creg == 0 && cnr == 0) {
          switch (dreg0 == 0xFF ? NRB : int(dreg0)) {
#define NQ_D1(B, _) case B: if constexpr (B <= NRB) rb_d1<C, NA, B, NRB>(a, m[0], m[1], tb); break;
            NQ_REG_CASES(NQ_D1, 0)
            case 5: if constexpr (NRB == 5) rb_d1<C, NA, 5, NRB>(a, m[0], m[1], tb); break;
#undef NQ_D1
            default: break;
          }
        } else {
          m[2] = m[0];
          m[3] = m[1];
          rb_diag_generic<C, NA>(a, m, 1, dreg0, 0xFF, tb, 0, tc, creg);
        }
        break;
      }
      case OP_D2: {
        C m[4] = {pm0, pm1, pm2, pm3};
        const uint32_t tb0 = (vbase & dv0) ? 1u : 0u;
        const uint32_t tb1 = (vbase & dv1) ? 1u : 0u;
        if (creg == 0 && cnr == 0) {
          const int d0 = dreg0 == 0xFF ? NRB : int(dreg0);
          const int d1 = dreg1 == 0xFF ? NRB : int(dreg1);
          switch (d0) {
#define NQ_D2A(V) case V: if constexpr (V <= NRB) dispatch_d2_b<C, NA, NRB, V>(a, d1, m, tb0, tb1); break;
            NQ_D2A(0) NQ_D2A(1) NQ_D2A(2) NQ_D2A(3) NQ_D2A(4) NQ_D2A(5)
#undef NQ_D2A
            default: break;
          }
        } else {
          rb_diag_generic<C, NA>(a, m, 2, dreg0, dreg1, tb0, tb1, tc, creg);
        }
        break;
      }
      case OP_U2: {
        switch (rb0) {
#define NQ_U2A(B, _) case B: if constexpr (B < NRB) dispatch_u2_b<Real, C, NA, NRB, B>(a, rb1, mp, tc, creg); break;
          NQ_REG_CASES(NQ_U2A, 0)
#undef NQ_U2A
          default: break;
        }
        break;
      }
      case OP_SW: {
        switch (rb0) {
#define NQ_SWA(B, _) case B: if constexpr (B < NRB) dispatch_sw_b<C, NA, NRB, B>(a, rb1, tc, creg); break;
          NQ_REG_CASES(NQ_SWA, 0)
#undef NQ_SWA
          default: break;
        }
        break;
      }
      default:
        break;
    }
  }
}

template <typename Real>
__device__ __forceinline__ void unpack_vec(const typename Tr<Real>::V& v, typename Tr<Real>::C* a);
template <>
__device__ __forceinline__ void unpack_vec<float>(const float4& v, float2* a) {
  a[0] = make_float2(v.x, v.y);
  a[1] = make_float2(v.z, v.w);
}
template <>
__device__ __forceinline__ void unpack_vec<double>(const double2& v, double2* a) {
  a[0] = v;
}
template <typename Real>
__device__ __forceinline__ typename Tr<Real>::V pack_vec(const typename Tr<Real>::C* a);
template <>
__device__ __forceinline__ float4 pack_vec<float>(const float2* a) {
  return make_float4(a[0].x, a[0].y, a[1].x, a[1].y);
}
template <>
__device__ __forceinline__ double2 pack_vec<double>(const double2* a) {
  return a[0];
}
template <typename Real>
__device__ __forceinline__ typename Tr<Real>::V pack_vec(typename Tr<Real>::C lo, typename Tr<Real>::C hi) {
  typename Tr<Real>::C t[2] = {lo, hi};
  return pack_vec<Real>(t);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Global amplitude index of tile-local index 0 of `tile` (tile id bit j -> qout[j]).
__device__ __forceinline__ uint64_t tile_base(const PassRec& P, uint64_t tile) {
  uint64_t base = 0;
  for (int j = 0; j < P.n_out; ++j)
    if ((tile >> j) & 1ull) base |= 1ull << P.qout[j];
  return base;
}


// Per-stage constants derived from a StageRec, kept in shared memory for the
// whole pass (kStageTabWords words per stage; built once per pass by
// build_stage_tab, so the per-tile stage loop does no bit-by-bit work):
//   S..S+3     slot offsets swz(vector bit of free register bit i)
//   CW..CW+3   slot offsets of the write-back images of the free register bits
//   HB         bit i: the image of free register bit i flips amplitude bit 0 (complex64)
//   MZ         image of register bit 0 (complex64; 1 = bit 0 stays bit 0)
//   CZ, HZ     slot offset and bit 0 of MZ's image
//   WS, WH     slot offset and bit 0 of the constant translation sbx
//   NC, OB, OE conditional translations, op range
//   CC, CS, CH per conditional translation: control mask, slot offset, bit 0
//   UL, UH     deposit of thread-index bits 0..3 / 4..7 into the vector index
//   SL, SH     the same deposits through the swizzle (swz is linear over XOR)
struct StageTab {
  enum : int { S = 0, CW = 4, HB = 8, MZ = 9, CZ = 10, HZ = 11, WS = 12, WH = 13, NC = 14, OB = 15, OE = 16,
               CC = 17, CS = 21, CH = 25, UL = 32, UH = 48, SL = 64, SH = 80 };
};
static_assert(StageTab::SH + 16 <= kStageTabWords, "stage table layout");

template <int VB>
__device__ void build_stage_tab(const StageRec* __restrict__ S, uint32_t* __restrict__ t) {
  uint32_t s[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) s[i] = swz(1u << (S->rpos[i] - VB));
  auto regslot = [&](uint32_t m) {
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if ((m >> (VB + i)) & 1u) x ^= s[i];
    return x;
  };
  uint32_t hb = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t m = uint32_t(S->scol[VB + i]);
    t[StageTab::S + i] = s[i];
    t[StageTab::CW + i] = regslot(m);
    hb |= (VB == 1 ? (m & 1u) : 0u) << i;
  }
  const uint32_t mz = VB == 1 ? uint32_t(S->scol[0]) : 1u;
  t[StageTab::HB] = hb;
  t[StageTab::MZ] = mz;
  t[StageTab::CZ] = regslot(mz);
  t[StageTab::HZ] = VB == 1 ? (mz & 1u) : 0u;
  t[StageTab::WS] = regslot(uint32_t(S->sbx));
  t[StageTab::WH] = VB == 1 ? (uint32_t(S->sbx) & 1u) : 0u;
  t[StageTab::NC] = uint32_t(S->ncond);
  t[StageTab::OB] = uint32_t(S->op_begin);
  t[StageTab::OE] = uint32_t(S->op_end);
  for (int i = 0; i < kMaxCondPerm; ++i) {
    const uint32_t w = uint32_t(S->cond_w[i]);
    t[StageTab::CC + i] = S->cond_cnr[i];
    t[StageTab::CS + i] = regslot(w);
    t[StageTab::CH + i] = VB == 1 ? (w & 1u) : 0u;
  }
  const int ntb = S->n_tbits;
  for (int v = 0; v < 16; ++v) {
    uint32_t lo = 0, hi = 0;
    for (int j = 0; j < 4; ++j) {
      if (j < ntb && ((v >> j) & 1)) lo |= 1u << S->tpos[j];
      if (j + 4 < ntb && ((v >> j) & 1)) hi |= 1u << S->tpos[j + 4];
    }
    t[StageTab::UL + v] = lo;
    t[StageTab::UH + v] = hi;
    t[StageTab::SL + v] = swz(lo);
    t[StageTab::SH + v] = swz(hi);
  }
}

// Build the stage tables of pass P into `tabs` (every thread of the CTA calls
// it; it ends with a block barrier).
template <typename Real>
__device__ __forceinline__ void build_pass_tabs(const PassRec& P, const StageRec* __restrict__ stages,
                                                uint32_t* __restrict__ tabs) {
  const int nst = P.stage_end - P.stage_begin;
  for (int i = threadIdx.x; i < nst; i += blockDim.x)
    build_stage_tab<Tr<Real>::kVecBit>(stages + P.stage_begin + i, tabs + i * kStageTabWords);
  __syncthreads();
}

// Run stages [P.stage_begin, P.stage_end) of a pass on the tile held in shared
// memory `sv` (swizzled vector slots), with the pass's stage tables in `tabs`.
// Every thread of the CTA must call it (it contains block barriers); threads
// >= nvec/16 only take part in them.
template <typename Real, bool kDiagFlat = false>
__device__ __forceinline__ void run_tile_stages(typename Tr<Real>::V* __restrict__ sv, const PassRec& P,
                                                const uint32_t* __restrict__ tabs,
                                                const TileOp<Real>* __restrict__ ops, uint32_t ext) {
  using T = Tr<Real>;
  using C = typename T::C;
  constexpr int VB = T::kVecBit;
  constexpr int APV = T::kAmpsPerVec;
  constexpr int NA = kVecPerThread * APV;
  constexpr int NRB = VB + kRegFree;
  const int tid = threadIdx.x;
  const uint32_t active_threads = (1u << (P.k - VB)) / kVecPerThread;
  const int nst = P.stage_end - P.stage_begin;
  for (int si = 0; si < nst; ++si) {
    const uint32_t* Tb = tabs + si * kStageTabWords;
    if (uint32_t(tid) < active_threads) {
      const uint32_t ub = Tb[StageTab::UL + (tid & 15)] | Tb[StageTab::UH + (tid >> 4)];
      // swz is linear over XOR and ub, vm_i have disjoint bits, so
      // swz(ub | sum vm_i) = swz(ub) ^ xor_i swz(vm_i).
      const uint32_t sb = Tb[StageTab::SL + (tid & 15)] ^ Tb[StageTab::SH + (tid >> 4)];
      const uint4 sq = *reinterpret_cast<const uint4*>(Tb + StageTab::S);
      const uint32_t s0 = sq.x, s1 = sq.y, s2 = sq.z, s3 = sq.w;
      C a[NA];
#pragma unroll
      for (int r = 0; r < kVecPerThread; ++r) {
        const uint32_t slot = sb ^ ((r & 1) ? s0 : 0u) ^ ((r & 2) ? s1 : 0u) ^
                              ((r & 4) ? s2 : 0u) ^ ((r & 8) ? s3 : 0u);
        unpack_vec<Real>(sv[slot], a + r * APV);
      }
      const uint32_t vbase = (ub << VB) | ext;
      apply_stage_ops<Real, NA, NRB, kDiagFlat>(a, ops, int(Tb[StageTab::OB]), int(Tb[StageTab::OE]), vbase);
      // Write-back through the stage's deferred permutation pi(p) = A p ^ w:
      // register amplitude p goes to the slot of logical index pi(p).  Slot
      // offsets are linear in the free register bits (register bits
      // VB..VB+3); for complex64, bit 0 of pi(p) selects the 8-byte half.
      uint32_t wslot = Tb[StageTab::WS], hw = Tb[StageTab::WH];
      const int nc = int(Tb[StageTab::NC]);
      for (int i = 0; i < nc; ++i) {
        const uint32_t cm = Tb[StageTab::CC + i];
        if ((vbase & cm) == cm) {
          wslot ^= Tb[StageTab::CS + i];
          hw ^= Tb[StageTab::CH + i];
        }
      }
      const uint4 cq = *reinterpret_cast<const uint4*>(Tb + StageTab::CW);
      const uint32_t c0 = cq.x, c1 = cq.y, c2 = cq.z, c3 = cq.w;
      const uint32_t sw = sb ^ wslot;
      if constexpr (VB == 1) {
        const uint32_t mz = Tb[StageTab::MZ], hb = Tb[StageTab::HB];
        const uint32_t h0 = hb & 1u, h1 = (hb >> 1) & 1u, h2 = (hb >> 2) & 1u, h3 = (hb >> 3) & 1u;
        if (mz == 1u) {
          // bit 0 stays bit 0: each vector keeps its pair, halves swap when
          // bit 0 of pi is flipped by the other register bits or by w
          if ((hb | hw) == 0u) {
            // no deferred flip of qubit 0 in this stage: whole vectors, no selects
#pragma unroll
            for (int r = 0; r < kVecPerThread; ++r) {
              const uint32_t slot = sw ^ ((r & 1) ? c0 : 0u) ^ ((r & 2) ? c1 : 0u) ^
                                    ((r & 4) ? c2 : 0u) ^ ((r & 8) ? c3 : 0u);
              sv[slot] = pack_vec<Real>(a[2 * r], a[2 * r + 1]);
            }
          } else {
#pragma unroll
            for (int r = 0; r < kVecPerThread; ++r) {
              const uint32_t slot = sw ^ ((r & 1) ? c0 : 0u) ^ ((r & 2) ? c1 : 0u) ^
                                    ((r & 4) ? c2 : 0u) ^ ((r & 8) ? c3 : 0u);
              const uint32_t hs = hw ^ ((r & 1) ? h0 : 0u) ^ ((r & 2) ? h1 : 0u) ^
                                  ((r & 4) ? h2 : 0u) ^ ((r & 8) ? h3 : 0u);
              const C lo = a[2 * r], hi = a[2 * r + 1];
              sv[slot] = hs ? pack_vec<Real>(hi, lo) : pack_vec<Real>(lo, hi);
            }
          }
        } else {
          // bit 0 moves into other bits: store each amplitude separately
          const uint32_t cz = Tb[StageTab::CZ], hz = Tb[StageTab::HZ];
          C* sa = reinterpret_cast<C*>(sv);
#pragma unroll
          for (int r = 0; r < kVecPerThread; ++r) {
            const uint32_t slot = sw ^ ((r & 1) ? c0 : 0u) ^ ((r & 2) ? c1 : 0u) ^
                                  ((r & 4) ? c2 : 0u) ^ ((r & 8) ? c3 : 0u);
            const uint32_t hs = hw ^ ((r & 1) ? h0 : 0u) ^ ((r & 2) ? h1 : 0u) ^
                                ((r & 4) ? h2 : 0u) ^ ((r & 8) ? h3 : 0u);
            sa[2 * slot + hs] = a[2 * r];
            sa[2 * (slot ^ cz) + (hs ^ hz)] = a[2 * r + 1];
          }
        }
      } else {
#pragma unroll
        for (int r = 0; r < kVecPerThread; ++r) {
          const uint32_t slot = sw ^ ((r & 1) ? c0 : 0u) ^ ((r & 2) ? c1 : 0u) ^
                                ((r & 4) ? c2 : 0u) ^ ((r & 8) ? c3 : 0u);
          sv[slot] = pack_vec<Real>(a + r * APV);
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace nqpu
