// Tiled multi-gate pass kernel (the plain method's main path).
//
// One launch = one HBM pass over the state: each CTA streams tiles of 2^k
// amplitudes (k <= 13 for complex64, 12 for complex128: 64 KB) from HBM into
// shared memory with coalesced 128-bit loads, applies every gate the planner
// assigned to the pass, and streams the tile back.  Gates run in register
// stages: each thread gathers 16 vectors (32 complex64 / 16 complex128
// amplitudes) that differ in the stage's register bits, applies all of the
// stage's ops with fully unrolled register code, and scatters them back.
//
// Reference semantics: each op performs the same per-amplitude arithmetic as
// GateOperations (R/lib.rs:617-1735) — 2x2 rows a*x + b*y for dense 1q gates
// (apply_unitary_pair_indexed, R/lib.rs:634), 4x4 rows for u2 (R/lib.rs:1536),
// swaps for X/CNOT/SWAP (R/lib.rs:712/835/1207) and phases for diagonal gates —
// in the state's own precision.
//
// Shared-memory layout: vector u (16 B) lives at slot swz(u) = u ^ fold3(u>>3)
// so that the 8 lanes of a quarter-warp that the planner maps to vector bits of
// distinct residue mod 3 hit 8 distinct 16-byte bank groups.
#include "sv_device.cuh"
#include "kernels.h"

namespace nqpu {

constexpr int kTileThreads = 256;
constexpr int kVecPerThread = 16;

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

// ---- register-block op bodies (B, B0, B1 are register-bit indices) --------

template <typename C, int NA, int B, bool CTRL>
__device__ __forceinline__ void rb_u1(C (&a)[NA], const C* m, bool tc, uint32_t creg) {
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    if (i & (1 << B)) continue;
    const int j = i | (1 << B);
    C x = a[i], y = a[j];
    C nx = cmac2(m[0], x, m[1], y);
    C ny = cmac2(m[2], x, m[3], y);
    if (CTRL) {
      const bool cond = tc && ((uint32_t(i) & creg) == creg);
      a[i] = csel(cond, nx, x);
      a[j] = csel(cond, ny, y);
    } else {
      a[i] = nx;
      a[j] = ny;
    }
  }
}

template <typename C, int NA, int B>
__device__ __forceinline__ void rb_x1(C (&a)[NA], bool tc, uint32_t creg) {
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    if (i & (1 << B)) continue;
    const int j = i | (1 << B);
    const bool cond = tc && ((uint32_t(i) & creg) == creg);
    C x = a[i], y = a[j];
    a[i] = csel(cond, y, x);
    a[j] = csel(cond, x, y);
  }
}

template <typename C, int NA, int B0, int B1>
__device__ __forceinline__ void rb_u2(C (&a)[NA], const C* m, bool tc, uint32_t creg) {
  constexpr int M0 = 1 << B0, M1 = 1 << B1;
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    if (i & (M0 | M1)) continue;
    const bool cond = tc && ((uint32_t(i) & creg) == creg);
    C x0 = a[i], x1 = a[i | M0], x2 = a[i | M1], x3 = a[i | M0 | M1];
    C y0 = cmac4(m + 0, x0, x1, x2, x3);
    C y1 = cmac4(m + 4, x0, x1, x2, x3);
    C y2 = cmac4(m + 8, x0, x1, x2, x3);
    C y3 = cmac4(m + 12, x0, x1, x2, x3);
    a[i] = csel(cond, y0, x0);
    a[i | M0] = csel(cond, y1, x1);
    a[i | M1] = csel(cond, y2, x2);
    a[i | M0 | M1] = csel(cond, y3, x3);
  }
}

template <typename C, int NA, int B0, int B1>
__device__ __forceinline__ void rb_sw(C (&a)[NA], bool tc, uint32_t creg) {
  constexpr int M0 = 1 << B0, M1 = 1 << B1;
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    if (i & (M0 | M1)) continue;
    const bool cond = tc && ((uint32_t(i) & creg) == creg);
    C x1 = a[i | M0], x2 = a[i | M1];
    a[i | M0] = csel(cond, x2, x1);
    a[i | M1] = csel(cond, x1, x2);
  }
}

// Dispatch a runtime register bit to a compile-time template argument.
#define NQ_CASE1(FN, B, ...) case B: if constexpr (B < NRB) FN<C, NA, B>(__VA_ARGS__); break;
#define NQ_SWITCH1(FN, BV, ...)                                        \
  switch (BV) {                                                        \
    NQ_CASE1(FN, 0, __VA_ARGS__) NQ_CASE1(FN, 1, __VA_ARGS__)          \
    NQ_CASE1(FN, 2, __VA_ARGS__) NQ_CASE1(FN, 3, __VA_ARGS__)          \
    NQ_CASE1(FN, 4, __VA_ARGS__) default: break;                       \
  }

template <typename C, int NA, int NRB, int B0, template <typename, int, int, int> class F>
struct Dummy {};

template <typename C, int NA, int NRB, int B0>
__device__ __forceinline__ void rb_u2_b1(int b1, C (&a)[NA], const C* m, bool tc, uint32_t creg) {
  switch (b1) {
#define NQ_U2C(B1) case B1: if constexpr (B1 < NRB && B1 != B0) rb_u2<C, NA, B0, B1>(a, m, tc, creg); break;
    NQ_U2C(0) NQ_U2C(1) NQ_U2C(2) NQ_U2C(3) NQ_U2C(4)
#undef NQ_U2C
    default: break;
  }
}
template <typename C, int NA, int NRB, int B0>
__device__ __forceinline__ void rb_sw_b1(int b1, C (&a)[NA], bool tc, uint32_t creg) {
  switch (b1) {
#define NQ_SWC(B1) case B1: if constexpr (B1 < NRB && B1 != B0) rb_sw<C, NA, B0, B1>(a, tc, creg); break;
    NQ_SWC(0) NQ_SWC(1) NQ_SWC(2) NQ_SWC(3) NQ_SWC(4)
#undef NQ_SWC
    default: break;
  }
}

template <typename Real>
__device__ __forceinline__ void load_matrix(const Real* __restrict__ src, typename Tr<Real>::C* m, int count) {
  for (int i = 0; i < count; ++i) {
    m[i].x = __ldg(src + 2 * i);
    m[i].y = __ldg(src + 2 * i + 1);
  }
}

// Apply ops [ob, oe) of a stage to the thread's register block.
// vbase = virtual index of register amplitude 0 (register bits are zero in it).
template <typename Real, int NA, int NRB>
__device__ __forceinline__ void apply_stage_ops(typename Tr<Real>::C (&a)[NA],
                                                const TileOp<Real>* __restrict__ ops, int ob,
                                                int oe, uint32_t vbase) {
  using C = typename Tr<Real>::C;
  for (int o = ob; o < oe; ++o) {
    const TileOp<Real>* op = ops + o;
    const uint4 h0 = __ldg(reinterpret_cast<const uint4*>(op));
    const uint4 h1 = __ldg(reinterpret_cast<const uint4*>(op) + 1);
    const uint32_t kind = h0.x & 0xFF;
    const uint32_t rb0 = (h0.x >> 8) & 0xFF;
    const uint32_t rb1 = (h0.x >> 16) & 0xFF;
    const uint32_t creg = (h0.x >> 24) & 0xFF;
    const uint32_t dreg0 = h0.y & 0xFF;
    const uint32_t dreg1 = (h0.y >> 8) & 0xFF;
    const uint32_t cnr = h0.z;
    const uint32_t dv0 = h0.w;
    const uint32_t dv1 = h1.x;
    const bool tc = (vbase & cnr) == cnr;
    const Real* mp = op->m;
    C m[16];
    switch (kind) {
      case OP_U1: {
        load_matrix<Real>(mp, m, 4);
        if (cnr == 0 && creg == 0) {
          switch (rb0) {
#define NQ_U1N(B) case B: if constexpr (B < NRB) rb_u1<C, NA, B, false>(a, m, tc, creg); break;
            NQ_U1N(0) NQ_U1N(1) NQ_U1N(2) NQ_U1N(3) NQ_U1N(4)
#undef NQ_U1N
            default: break;
          }
        } else {
          switch (rb0) {
#define NQ_U1C(B) case B: if constexpr (B < NRB) rb_u1<C, NA, B, true>(a, m, tc, creg); break;
            NQ_U1C(0) NQ_U1C(1) NQ_U1C(2) NQ_U1C(3) NQ_U1C(4)
#undef NQ_U1C
            default: break;
          }
        }
        break;
      }
      case OP_X1: {
        switch (rb0) {
#define NQ_X1(B) case B: if constexpr (B < NRB) rb_x1<C, NA, B>(a, tc, creg); break;
          NQ_X1(0) NQ_X1(1) NQ_X1(2) NQ_X1(3) NQ_X1(4)
#undef NQ_X1
          default: break;
        }
        break;
      }
      case OP_U2: {
        load_matrix<Real>(mp, m, 16);
        switch (rb0) {
#define NQ_U2A(B0) case B0: if constexpr (B0 < NRB) rb_u2_b1<C, NA, NRB, B0>(rb1, a, m, tc, creg); break;
          NQ_U2A(0) NQ_U2A(1) NQ_U2A(2) NQ_U2A(3) NQ_U2A(4)
#undef NQ_U2A
          default: break;
        }
        break;
      }
      case OP_SW: {
        switch (rb0) {
#define NQ_SWA(B0) case B0: if constexpr (B0 < NRB) rb_sw_b1<C, NA, NRB, B0>(rb1, a, tc, creg); break;
          NQ_SWA(0) NQ_SWA(1) NQ_SWA(2) NQ_SWA(3) NQ_SWA(4)
#undef NQ_SWA
          default: break;
        }
        break;
      }
      case OP_D1: {
        load_matrix<Real>(mp, m, 2);
        const uint32_t tb = (vbase & dv0) ? 1u : 0u;
#pragma unroll
        for (int i = 0; i < NA; ++i) {
          const bool cond = tc && ((uint32_t(i) & creg) == creg);
          const uint32_t b = (dreg0 != 0xFF) ? ((uint32_t(i) >> dreg0) & 1u) : tb;
          const C d = csel(b != 0, m[1], m[0]);
          a[i] = csel(cond, cmul(d, a[i]), a[i]);
        }
        break;
      }
      case OP_D2: {
        load_matrix<Real>(mp, m, 4);
        const uint32_t tb0 = (vbase & dv0) ? 1u : 0u;
        const uint32_t tb1 = (vbase & dv1) ? 1u : 0u;
#pragma unroll
        for (int i = 0; i < NA; ++i) {
          const bool cond = tc && ((uint32_t(i) & creg) == creg);
          const uint32_t b0 = (dreg0 != 0xFF) ? ((uint32_t(i) >> dreg0) & 1u) : tb0;
          const uint32_t b1 = (dreg1 != 0xFF) ? ((uint32_t(i) >> dreg1) & 1u) : tb1;
          const C lo = csel(b0 != 0, m[1], m[0]);
          const C hi = csel(b0 != 0, m[3], m[2]);
          const C d = csel(b1 != 0, hi, lo);
          a[i] = csel(cond, cmul(d, a[i]), a[i]);
        }
        break;
      }
      case OP_PH: {
        load_matrix<Real>(mp, m, 1);
#pragma unroll
        for (int i = 0; i < NA; ++i) {
          const bool cond = tc && ((uint32_t(i) & creg) == creg);
          a[i] = csel(cond, cmul(m[0], a[i]), a[i]);
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

// Dynamic shared memory: [vectors of the tile | hi_off table (2^(k-c) u64)].
template <typename Real, int KMAX>
__global__ void __launch_bounds__(kTileThreads, 2)
    k_tile_pass(Real* __restrict__ amp, const PassRec* __restrict__ passes,
                const StageRec* __restrict__ stages, const TileOp<Real>* __restrict__ ops,
                int pass_idx, uint64_t n_tiles) {
  using T = Tr<Real>;
  using C = typename T::C;
  using V = typename T::V;
  constexpr int VB = T::kVecBit;
  constexpr int APV = T::kAmpsPerVec;
  constexpr int NA = kVecPerThread * APV;  // amplitudes per thread
  constexpr int NRB = VB + kRegFree;       // register bits
  constexpr uint32_t kMaxVec = 1u << (KMAX - VB);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* sv = reinterpret_cast<V*>(smem_raw);
  uint64_t* hi_off = reinterpret_cast<uint64_t*>(smem_raw + sizeof(V) * kMaxVec);
  __shared__ PassRec P;

  const int tid = threadIdx.x;
  {
    const int32_t* src = reinterpret_cast<const int32_t*>(passes + pass_idx);
    int32_t* dst = reinterpret_cast<int32_t*>(&P);
    for (int i = tid; i < int(sizeof(PassRec) / 4); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int k = P.k, c = P.c;
  const uint32_t nvec = 1u << (k - VB);
  const int nhi = k - c;
  for (int h = tid; h < (1 << nhi); h += blockDim.x) {
    uint64_t off = 0;
    for (int j = 0; j < nhi; ++j)
      if ((h >> j) & 1) off |= 1ull << P.qhi[j];
    hi_off[h] = off;
  }
  __syncthreads();
  const uint32_t lowmask = (1u << c) - 1u;
  const uint32_t active_threads = nvec / kVecPerThread;

  for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    uint64_t base = 0;
    for (int j = 0; j < P.n_out; ++j)
      if ((tile >> j) & 1ull) base |= 1ull << P.qout[j];
    uint32_t ext = 0;
    for (int j = 0; j < P.n_ext; ++j)
      if ((base >> P.ext[j]) & 1ull) ext |= 1u << (k + j);

    // HBM -> shared (coalesced: consecutive threads take consecutive vectors).
    {
      V tmp[kVecPerThread];
#pragma unroll
      for (int i = 0; i < kVecPerThread; ++i) {
        const uint32_t u = tid + i * kTileThreads;
        if (u < nvec) {
          const uint32_t t = u << VB;
          const uint64_t g = base + (t & lowmask) + hi_off[t >> c];
          tmp[i] = __ldcs(reinterpret_cast<const V*>(amp + 2 * g));
        }
      }
#pragma unroll
      for (int i = 0; i < kVecPerThread; ++i) {
        const uint32_t u = tid + i * kTileThreads;
        if (u < nvec) sv[swz(u)] = tmp[i];
      }
    }
    __syncthreads();

    for (int s = P.stage_begin; s < P.stage_end; ++s) {
      const StageRec* S = stages + s;
      if (uint32_t(tid) < active_threads) {
        const int ntb = __ldg(&S->n_tbits);
        uint32_t ub = 0;
        for (int j = 0; j < ntb; ++j) ub |= ((uint32_t(tid) >> j) & 1u) << __ldg(&S->tpos[j]);
        const uint32_t vm0 = 1u << (__ldg(&S->rpos[0]) - VB);
        const uint32_t vm1 = 1u << (__ldg(&S->rpos[1]) - VB);
        const uint32_t vm2 = 1u << (__ldg(&S->rpos[2]) - VB);
        const uint32_t vm3 = 1u << (__ldg(&S->rpos[3]) - VB);
        C a[NA];
#pragma unroll
        for (int r = 0; r < kVecPerThread; ++r) {
          const uint32_t u = ub | ((r & 1) ? vm0 : 0u) | ((r & 2) ? vm1 : 0u) |
                             ((r & 4) ? vm2 : 0u) | ((r & 8) ? vm3 : 0u);
          unpack_vec<Real>(sv[swz(u)], a + r * APV);
        }
        const uint32_t vbase = (ub << VB) | ext;
        apply_stage_ops<Real, NA, NRB>(a, ops, __ldg(&S->op_begin), __ldg(&S->op_end), vbase);
#pragma unroll
        for (int r = 0; r < kVecPerThread; ++r) {
          const uint32_t u = ub | ((r & 1) ? vm0 : 0u) | ((r & 2) ? vm1 : 0u) |
                             ((r & 4) ? vm2 : 0u) | ((r & 8) ? vm3 : 0u);
          sv[swz(u)] = pack_vec<Real>(a + r * APV);
        }
      }
      __syncthreads();
    }

    // shared -> HBM
#pragma unroll
    for (int i = 0; i < kVecPerThread; ++i) {
      const uint32_t u = tid + i * kTileThreads;
      if (u < nvec) {
        const uint32_t t = u << VB;
        const uint64_t g = base + (t & lowmask) + hi_off[t >> c];
        __stcs(reinterpret_cast<V*>(amp + 2 * g), sv[swz(u)]);
      }
    }
    __syncthreads();
  }
}

template <typename Real>
static int tile_kmax() {
  return sizeof(Real) == 4 ? 13 : 12;
}

template <typename Real>
static size_t tile_smem_bytes() {
  using V = typename Tr<Real>::V;
  const int kmax = tile_kmax<Real>();
  return sizeof(V) * (size_t(1) << (kmax - Tr<Real>::kVecBit)) + sizeof(uint64_t) * 1024;
}

template <typename Real>
cudaError_t launch_tile_pass_t(Real* amp, int n, const PassRec& host_pass, const PassRec* d_passes,
                               const StageRec* d_stages, const TileOp<Real>* d_ops, int pass_idx,
                               cudaStream_t stream, int num_sms) {
  constexpr int KMAX = sizeof(Real) == 4 ? 13 : 12;
  auto kern = k_tile_pass<Real, KMAX>;
  const size_t smem = tile_smem_bytes<Real>();
  static bool configured[2] = {false, false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!configured[sizeof(Real) == 4 ? 0 : 1]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    configured[sizeof(Real) == 4 ? 0 : 1] = true;
  }
  (void)n;
  const uint64_t n_tiles = 1ull << host_pass.n_out;
  const uint64_t max_ctas = uint64_t(num_sms) * 2;
  const unsigned grid = unsigned(n_tiles < max_ctas ? n_tiles : max_ctas);
  kern<<<grid, kTileThreads, smem, stream>>>(amp, d_passes, d_stages, d_ops, pass_idx, n_tiles);
  return cudaGetLastError();
}

cudaError_t launch_tile_pass(DType dt, void* amp, int n, const PassRec& host_pass,
                             const PassRec* d_passes, const StageRec* d_stages, const void* d_ops,
                             int pass_idx, cudaStream_t stream, int num_sms) {
  if (dt == DType::C64)
    return launch_tile_pass_t<float>(static_cast<float*>(amp), n, host_pass, d_passes, d_stages,
                                     static_cast<const TileOp<float>*>(d_ops), pass_idx, stream,
                                     num_sms);
  return launch_tile_pass_t<double>(static_cast<double*>(amp), n, host_pass, d_passes, d_stages,
                                    static_cast<const TileOp<double>*>(d_ops), pass_idx, stream,
                                    num_sms);
}

int tile_kmax_for(DType dt) { return dt == DType::C64 ? 13 : 12; }

}  // namespace nqpu
