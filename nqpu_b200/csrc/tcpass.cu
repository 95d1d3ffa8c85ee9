// Tensor-core pass mode (complex64): several fused 5-qubit unitaries per HBM
// pass, each applied as a tcgen05 GEMM with split FP16 operands on a tile held
// in shared memory (plan data and layouts in tcpass.h, planner in tcplan.cpp).
//
// Per pass, one persistent CTA per SM with five independent tile engines of
// four warps (one per TMEM lane quadrant).  An engine owns an operand buffer
// (the tile as the 128 x 64 FP16 A operand: hi and lo planes, K-major,
// 128-byte swizzle, 32 KB) and a 64-column TMEM accumulator, and runs its
// tiles through:
//   load     the tile's 32 KB (256 runs of 16 contiguous amplitudes) arrive
//            by 16-byte cp.async as raw FP32 in the engine's own operand
//            buffer, at the plan's landing offsets (tcpass.h:
//            tc_raw_offsets); they are issued as soon as the previous tile's
//            last MMAs are done, so they fly during that tile's last epilogue;
//   split    in two halves (load-step bit 3 = 0, 1), each landed in the
//            slots that only its own outputs fill: each thread reads back its
//            own 8 chunks of the half, the engine meets at a barrier (the
//            buffer is converted in place), then scales by s (a power of two,
//            for the FP16 range) and the renormalisation factor, splits
//            x = hi + lo into FP16 pairs and stores them in unitary 0's
//            operand layout (half the raw tile in registers at a time is what
//            lets five engines run at 96 registers);
//   unitary  one elected thread issues 12 MMAs (K = 16, N = 64) into the
//            engine's 64-column accumulator: D = A_hi B_hi^T + A_hi B_lo^T +
//            A_lo B_hi^T, B = the real embedding of 16 U, and commits them to
//            the engine's mbarrier; one warp polls it (bounded) while the
//            other three wait at the engine's named barrier;
//   epilogue each thread drains its row (TMEM lane) of D, two 4-column parts
//            per TMEM load wait, forms out = D / 16 and either splits it
//            straight into the next unitary's operand layout, or, after the
//            last unitary, stores out / s to HBM; there, up to two
//            warp-shuffle exchanges of a lane bit with a column bit first put
//            the state's low index bits on lanes, so a warp store covers
//            whole 128-byte lines (3.75 lines per store on the 30-qubit
//            brickwork instead of 9.9; 6-7 % of the circuit's time).
// While one engine waits for its MMAs the other four run, so the tensor
// pipe, shared memory and HBM overlap across five tiles.  The B operands of
// the pass's unitaries stay in shared memory for the launch.  The stores
// follow the pass's store-side index bits (qt_out), which may place the tile's
// qubits on other state index bits than it loaded them from (see tcpass.h).
//
// Renormalisation: the first pass of a run records the FP64 norm of its input
// (per-CTA partials) and every pass the norm of its output; each later pass
// scales its input by sqrt(norm_in / norm_prev_out), so the norm drift of the
// split-precision contractions is removed without an extra HBM pass and the
// state keeps the norm it had when the run started.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "device_once.h"
#include "engine.h"
#include "kernels.h"
#include "tcpass.h"
#include "tcrun.h"
#include "umma.cuh"

namespace nqpu {

// An engine is one warp per TMEM lane quadrant (4 warps, 128 threads): each
// thread drains whole rows, so 640 threads per CTA with up to 96 registers
// each.  (Measured on the 30-qubit brickwork: 4-warp engines against 8-warp
// ones with two warps per quadrant at 64 registers, 2-3.5 % faster; five
// engines with the two-phase split against four with the whole raw tile in
// registers, about 1 % faster — the split's second barrier costs 2.5 %, the
// fifth engine gains 3.5 %.)
constexpr int kTcEngines = 5;
constexpr int kTcEngineWarps = 4;
constexpr int kTcEngineThreads = 32 * kTcEngineWarps;
constexpr int kTcThreads = kTcEngines * kTcEngineThreads;
constexpr int kTcThrBits = kTcLoadThreadBits;                 // loader: thread bits of an engine
constexpr int kTcStpBits = kTcLoadStepBits;                   // loader: step bits
static_assert((1 << kTcThrBits) == kTcEngineThreads, "one loading thread per engine thread");
static_assert(kTcThrBits + kTcStpBits == kTcTileBits - 1, "loads cover the tile");
constexpr int kTcLoadSteps = 1 << kTcStpBits;                 // 16-byte chunks per thread per tile
constexpr int kTcColHalves = kTcEngineWarps / 4;              // warps sharing a lane quadrant
constexpr int kTcCols = 32 / kTcColHalves;                    // complex columns a thread drains
constexpr int kTcParts = kTcCols / 4;                         // epilogue parts of 4 columns
// All three split products accumulate into one 64-column accumulator (12
// MMAs of N = 64).  (Measured against A_hi [B_hi; B_lo]^T with N = 128 plus
// A_lo B_hi^T into 128 columns summed in the epilogue: the same speed, half
// the infidelity, half the TMEM loads.)  Two parts per TMEM load wait keep
// the five engines' drain within 96 registers.
constexpr int kTcBatch = 2;                                   // parts per TMEM load wait
constexpr uint32_t kTcAccCols = 64;                           // accumulator columns per engine
static_assert(kTcEngines * kTcAccCols <= 512, "accumulators fit tensor memory");
static_assert(kTcParts % kTcBatch == 0, "whole batches");
constexpr uint32_t kTcAPlane = 128 * 128;            // 16 KB: 128 rows x 64 halves
constexpr uint32_t kTcOpBytes = 2 * kTcAPlane;       // hi + lo planes
constexpr uint32_t kTcBBytes = 128 * 128;            // [B_hi; B_lo]: 128 rows x 64 halves
constexpr uint32_t kTcWaitLimit = 1u << 22;          // bounded mbarrier polls (default)
constexpr uint32_t kTcTmemCols = 512;                // the engines' accumulators (allocated as a power of two)

// Every offset the kernel forms is GF(2)-linear in the bits of its index (the
// swizzled operand layout XORs disjoint fields; amplitude offsets OR disjoint
// qubit bits), so the tables hold one entry per index bit and the kernel
// combines them with XORs / adds of compile-time selections.
struct TcTables {
  uint32_t xcb[kTcMaxUnitaries][5];  // epilogue of unitary j: next-layout operand offset of column bit i
  uint64_t gcb[kTcMaxUnitaries][5];  // epilogue of the last unitary: amplitude offset of column bit i
  uint32_t sob[kTcStpBits];          // loader: operand offset (unitary 0's layout) of step bit s
  uint32_t rsb[kTcStpBits];          // loader: raw landing offset of step bit s
  uint64_t sgb[kTcStpBits];          // loader: amplitude offset of step bit s
};

constexpr size_t kTcSmem = 1024 /*alignment*/ + kTcEngines * size_t(kTcOpBytes) +
                           kTcMaxUnitaries * size_t(kTcBBytes) + sizeof(TcTables);
static_assert(kTcSmem <= 232448, "dynamic shared memory of one CTA");

constexpr uint32_t kIdescN64 = umma_idesc_f16<128, 64>();

__device__ __forceinline__ void engine_sync(int e) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(1 + e), "n"(kTcEngineThreads) : "memory");
}

__device__ __forceinline__ float4 lds_v4(uint32_t addr) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(addr)
               : "memory");
  return v;
}
__device__ __forceinline__ void cp_async16_s(uint32_t saddr, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// FP16 hi/lo split of an (re, im) pair: hi = half(x), lo = half(x - hi)
// (x - hi is exact in FP32; one packed FP32x2 FMA), as two packed half2 words.
__device__ __forceinline__ void split_pair(float2 x, uint32_t& hi, uint32_t& lo) {
  const __half2 h = __float22half2_rn(x);
  const float2 r = __ffma2_rn(__half22float2(h), make_float2(-1.0f, -1.0f), x);
  const __half2 l = __float22half2_rn(r);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// Last epilogue: exchange lane bit l (lmask = 1 << l) with column bit KC of a
// 16-column batch across the warp.  Lane t's register of column c then holds
// the element of lane t with bit l set to c's bit KC, column c with bit KC set
// to t's bit l: the lane with bit l set sends its column of bit KC = 0 and
// takes its partner's column of bit KC = 1 in its place, the partner the
// reverse (one shuffle per register pair).
static_assert(4 * kTcBatch >= (2 << kTcMaxLaneSwaps) && kTcColHalves == 1,
              "lane exchanges: column bits 1..kTcMaxLaneSwaps inside a batch, one thread per row");
template <int KC>
__device__ __forceinline__ void lane_swap(uint32_t (&rh)[kTcBatch][8], uint32_t lmask, bool up) {
#pragma unroll
  for (int c = 0; c < 4 * kTcBatch; ++c) {
    if (c & (1 << KC)) continue;
    const int c2 = c | (1 << KC);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint32_t& a = rh[c >> 2][2 * (c & 3) + h];
      uint32_t& b = rh[c2 >> 2][2 * (c2 & 3) + h];
      const uint32_t r = __shfl_xor_sync(0xffffffffu, up ? a : b, lmask);
      if (up) a = r;
      else b = r;
    }
  }
}

__global__ void __launch_bounds__(kTcThreads, 1)
    k_tc_pass(float* __restrict__ amp, const TcPassRec* __restrict__ pass, const uint16_t* __restrict__ bmats,
              uint32_t n_tiles, float state_scale, const double* __restrict__ norm0,
              double* __restrict__ norm0_out, const double* __restrict__ prev_norm, int n_prev,
              double* __restrict__ out_norm, int* __restrict__ err, uint32_t wait_limit) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw_s = static_cast<uint32_t>(__cvta_generic_to_shared(smem_raw));
  unsigned char* base_p = smem_raw + ((1024 - (raw_s & 1023)) & 1023);
  unsigned char* opbuf = base_p;                                    // [engine][hi | lo]
  unsigned char* bbuf = base_p + kTcEngines * kTcOpBytes;           // [unitary][128 rows x 64 halves]
  TcTables* T = reinterpret_cast<TcTables*>(bbuf + kTcMaxUnitaries * kTcBBytes);
  __shared__ TcPassRec P;
  __shared__ __align__(8) uint64_t mbar[kTcEngines];
  __shared__ __align__(8) uint64_t mbar_never;  // failure injection: a barrier nothing arrives on
  __shared__ uint32_t tmem_holder;
  __shared__ int s_abort[kTcEngines];
  __shared__ float s_scale_in;
  __shared__ double s_red[2][kTcThreads / 32];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int e = tid / kTcEngineThreads, et = tid % kTcEngineThreads;
  const int q = warp & 3, ch = (et >> 7) & (kTcColHalves - 1);  // TMEM lane quadrant, column half
  const uint32_t row = uint32_t(32 * q + lane);  // this thread's operand row = its TMEM lane

  // ---- prologue: pass record, B operands, tables, barriers, TMEM ----
  {
    const int32_t* src = reinterpret_cast<const int32_t*>(pass);
    int32_t* dst = reinterpret_cast<int32_t*>(&P);
    for (int i = tid; i < int(sizeof(TcPassRec) / 4); i += kTcThreads) dst[i] = __ldg(src + i);
  }
  __syncthreads();
  const int m = P.m;
  for (int j = 0; j < m; ++j) {
    // 8 halves (16 bytes) per copy: a 16-byte chunk of the swizzled row
    const uint4* bsrc = reinterpret_cast<const uint4*>(bmats + size_t(j) * kTcBmatHalves);
    unsigned char* bdst = bbuf + j * kTcBBytes;
    for (int i = tid; i < int(kTcBmatHalves / 8); i += kTcThreads) {
      const uint32_t nrow = uint32_t(i) >> 3, k = (uint32_t(i) & 7u) * 8u;
      *reinterpret_cast<uint4*>(bdst + tc_sw128_off(nrow, k)) = __ldg(bsrc + i);
    }
  }
  if (tid < 5 * m) {
    const int j = tid / 5, i = tid % 5;
    T->xcb[j][i] = j + 1 < m ? P.u[j + 1].boff[P.u[j].fcol[i]] : 0u;
    // the last epilogue's column bit 1 + s stores to the index bit of lane bit
    // sw_lane[s] after the lane exchange
    int sb = P.qt_out[P.u[j].fcol[i]];
    if (j + 1 == m && i >= 1 && i <= 3 && P.sw_lane[i - 1] >= 0) sb = P.qt_out[P.u[j].frow[P.sw_lane[i - 1]]];
    T->gcb[j][i] = 1ull << sb;
  }
  if (tid < kTcStpBits) {
    T->sob[tid] = P.u[0].boff[P.lt[kTcThrBits + tid]];
    T->rsb[tid] = P.roff[P.lt[kTcThrBits + tid]];
    T->sgb[tid] = 1ull << P.qt[P.lt[kTcThrBits + tid]];
  }
  const uint32_t mbar_s = static_cast<uint32_t>(__cvta_generic_to_shared(&mbar[0]));
  if (tid < kTcEngines) {
    mbar_init(mbar_s + 8u * uint32_t(tid), 1);
    s_abort[tid] = 0;
  }
  const uint32_t never_s = static_cast<uint32_t>(__cvta_generic_to_shared(&mbar_never));
  if (tid == 0) mbar_init(never_s, 1);
  // wait_limit: polls of the first MMA wait; bit 31 points that wait at
  // mbar_never, so it expires (tests of the error path)
  const bool inject = (wait_limit >> 31) != 0;
  const uint32_t first_limit = wait_limit & 0x7FFFFFFFu;
  if (warp == 0) {
    const uint32_t holder = static_cast<uint32_t>(__cvta_generic_to_shared(&tmem_holder));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(holder),
                 "r"(kTcTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (warp == 1) {
    // renormalisation factor of this pass's input, times the operand scale s:
    // one warp sums the per-CTA partials in a fixed order (every CTA gets the
    // same factor) and shares it
    float sc = state_scale;
    if (prev_norm && norm0) {
      double t0 = 0.0, tp = 0.0;
      for (int i = lane; i < n_prev; i += 32) {
        t0 += norm0[i];
        tp += prev_norm[i];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        t0 += __shfl_xor_sync(0xffffffffu, t0, o);
        tp += __shfl_xor_sync(0xffffffffu, tp, o);
      }
      if (t0 > 0.0 && tp > 0.0) sc = float(double(state_scale) * sqrt(t0 / tp));
    }
    if (lane == 0) s_scale_in = sc;
  }
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  fence_proxy_async_smem();  // the B operands, written by generic stores, are read by the tensor core
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_holder;

  const float scale_in = s_scale_in;
  const float mid_scale = 1.0f / kTcUScale;                       // exact: a power of two
  const float out_scale = 1.0f / (kTcUScale * state_scale);       // exact: a power of two

  // ---- per-thread address parts ----
  // loader: thread bit b of et is tile bit lt[b], step bit s is tile bit
  // lt[kTcThrBits + s], and tile bit 0 is the pair inside each 16-byte load
  uint32_t pol = 0, raw_t = 0;
  uint64_t pgl = 0;
  for (int b = 0; b < kTcThrBits; ++b)
    if ((et >> b) & 1) {
      pol ^= P.u[0].boff[P.lt[b]];
      raw_t ^= P.roff[P.lt[b]];
      pgl |= 1ull << P.qt[P.lt[b]];
    }
  const uint32_t boff_h = P.u[0].boff[0];
  const bool load_pair = boff_h == 4u;  // tile bit 0 is column bit 0: the two amplitudes are adjacent
  // epilogue of unitary j: row part of the thread's row (its TMEM lane)
  uint32_t ptn[kTcMaxUnitaries];
  bool pair[kTcMaxUnitaries];
  uint64_t pg = 0;
#pragma unroll
  for (int j = 0; j < kTcMaxUnitaries; ++j) {
    ptn[j] = 0;
    pair[j] = false;
    if (j + 1 < m) {
      for (int i = 0; i < 7; ++i)
        if ((row >> i) & 1u) ptn[j] ^= P.u[j + 1].boff[P.u[j].frow[i]];
      pair[j] = P.u[j + 1].boff[P.u[j].fcol[0]] == 4u;
    } else if (j + 1 == m) {
      for (int i = 0; i < 7; ++i)
        if ((row >> i) & 1u) {
          int sb = P.qt_out[P.u[j].frow[i]];
          for (int s = 0; s < 3; ++s)
            if (P.sw_lane[s] == i) sb = P.qt_out[P.u[j].fcol[1 + s]];  // exchanged with column bit 1 + s
          pg |= 1ull << sb;
        }
    }
  }
  const bool store16 = P.qt_out[P.u[m - 1].fcol[0]] == 0;  // index bit 0 is column bit 0 of the last layout

  const uint32_t ahi_s = static_cast<uint32_t>(__cvta_generic_to_shared(opbuf)) + uint32_t(e) * kTcOpBytes;
  const uint32_t alo_s = ahi_s + kTcAPlane;
  const uint32_t b_s = static_cast<uint32_t>(__cvta_generic_to_shared(bbuf));
  const uint32_t my_mbar = mbar_s + 8u * uint32_t(e);
  const uint32_t acc = tmem + kTcAccCols * uint32_t(e);
  const uint32_t lanes = acc + (uint32_t(q * 32) << 16) + uint32_t(2 * kTcCols * ch);

  auto tile_base_of = [&](uint32_t tile) {
    const uint64_t mine = (lane < P.n_out && ((tile >> lane) & 1u)) ? (1ull << P.qout[lane]) : 0ull;
    const uint32_t lo = __reduce_or_sync(0xffffffffu, uint32_t(mine));
    const uint32_t hi = __reduce_or_sync(0xffffffffu, uint32_t(mine >> 32));
    return uint64_t(lo) | (uint64_t(hi) << 32);
  };
  // split an amplitude (or two adjacent ones) into the hi / lo planes at byte offset o
  auto put1 = [&](uint32_t o, float2 x) {
    uint32_t h, l;
    split_pair(x, h, l);
    sts_b32(ahi_s + o, h);
    sts_b32(alo_s + o, l);
  };
  auto put2 = [&](uint32_t o, float2 x0, float2 x1) {
    uint32_t h0, l0, h1, l1;
    split_pair(x0, h0, l0);
    split_pair(x1, h1, l1);
    sts_v2_b32(ahi_s + o, h0, h1);
    sts_v2_b32(alo_s + o, l0, l1);
  };
  auto engine_barrier = [&]() {
    tc_fence_before();
    engine_sync(e);
    tc_fence_after();
  };
  // raw FP32 chunks of `tile` into the engine's operand buffer by 16-byte
  // cp.async: this thread's chunk of step i at raw_t ^ (the step bits' raw
  // offsets), in the 16-byte slots its own half of the split fills (the
  // plan's landing offsets); each thread reads back only its own chunks
  // (the step bits' entries are read from the shared tables where they are
  // used: no registers held across the drain or the split)
  auto raw_off = [&](int i) {
    uint32_t r = raw_t;
#pragma unroll
    for (int b = 0; b < kTcStpBits; ++b)
      if ((i >> b) & 1) r ^= T->rsb[b];
    return r;
  };
  auto issue_loads = [&](uint32_t tile) {
    const uint64_t tbn = tile_base_of(tile);
    const float4* src = reinterpret_cast<const float4*>(amp) + ((tbn + pgl) >> 1);
    uint64_t sgb[kTcStpBits];
#pragma unroll
    for (int b = 0; b < kTcStpBits; ++b) sgb[b] = T->sgb[b] >> 1;  // in 16-byte chunks
#pragma unroll
    for (int i = 0; i < kTcLoadSteps; ++i) {
      uint64_t a = 0;
#pragma unroll
      for (int b = 0; b < kTcStpBits; ++b)
        if ((i >> b) & 1) a += sgb[b];
      cp_async16_s(ahi_s + raw_off(i), src + a);
    }
    cp_async_commit();
  };

  double norm_in = 0.0, norm_out = 0.0;
  uint32_t phase = 0;  // parity of the engine's mbarrier phase to wait for
  const uint32_t stride = uint32_t(kTcEngines) * gridDim.x;
  const uint32_t first_tile = uint32_t(kTcEngines) * blockIdx.x + uint32_t(e);
  if (first_tile < n_tiles) issue_loads(first_tile);
  for (uint32_t tile = first_tile; tile < n_tiles; tile += stride) {
    const uint64_t tb = tile_base_of(tile);
    // ---- load, scale, split into unitary 0's operand ----
    {
      cp_async_wait0();
      uint32_t sob[kTcStpBits];
#pragma unroll
      for (int b = 0; b < kTcStpBits; ++b) sob[b] = T->sob[b];
      const float2 s2 = make_float2(scale_in, scale_in);
      // compile-time forms: 8-byte operand stores when the two amplitudes of
      // a chunk are adjacent columns, the input norm on the first pass only
      auto split = [&](auto pair_c, auto norm_c) {
        constexpr bool kPair = decltype(pair_c)::value;
        constexpr bool kNorm = decltype(norm_c)::value;
        float2 nin = make_float2(0.0f, 0.0f);  // FP32 partials over this thread's amplitudes, FP64 across tiles
        // two halves (load-step bit 3 = 0, 1): each half's raw chunks sit in
        // the slots that only its own outputs overwrite, so half the chunks
        // are in registers at a time
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          constexpr int kHalf = kTcLoadSteps / 2;
          float4 v[kHalf];
#pragma unroll
          for (int ii = 0; ii < kHalf; ++ii) v[ii] = lds_v4(ahi_s + raw_off(ii + h * kHalf));
          engine_sync(e);  // this half's raw chunks are in registers before its operand overwrites them
#pragma unroll
          for (int ii = 0; ii < kHalf; ++ii) {
            const int i = ii + h * kHalf;
            const float2 x0 = make_float2(v[ii].x, v[ii].y), x1 = make_float2(v[ii].z, v[ii].w);
            if constexpr (kNorm) nin = __ffma2_rn(x1, x1, __ffma2_rn(x0, x0, nin));
            uint32_t o = pol;
#pragma unroll
            for (int b = 0; b < kTcStpBits; ++b)
              if ((i >> b) & 1) o ^= sob[b];
            if constexpr (kPair) {
              put2(o, __fmul2_rn(x0, s2), __fmul2_rn(x1, s2));
            } else {
              put1(o, __fmul2_rn(x0, s2));
              put1(o ^ boff_h, __fmul2_rn(x1, s2));
            }
          }
        }
        if constexpr (kNorm) norm_in += double(nin.x) + double(nin.y);
      };
      if (load_pair) {
        if (norm0_out) split(std::true_type{}, std::true_type{});
        else split(std::true_type{}, std::false_type{});
      } else {
        if (norm0_out) split(std::false_type{}, std::true_type{});
        else split(std::false_type{}, std::false_type{});
      }
    }
    fence_proxy_async_smem();
    engine_barrier();
    bool aborted = false;
    for (int j = 0; j < m; ++j) {
      // ---- unitary j on the tensor cores: 12 MMAs of K = 16, N = 64 ----
      if (et == 0) {
        // the descriptors differ only in their start-address field (address
        // >> 4), which these offsets do not carry out of
        const uint64_t dhi = umma_desc_sw128(ahi_s), dlo = umma_desc_sw128(alo_s);
        const uint64_t dbj = umma_desc_sw128(b_s + uint32_t(j) * kTcBBytes);
#pragma unroll
        // D = A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T; B_lo = rows 64..127 of
        // the B buffer: 8 KB on, a whole number of 1 KB swizzle atoms (512 in
        // the descriptor's 16-byte units)
        for (int kk = 0; kk < 4; ++kk) umma_f16(acc, dhi + 2u * kk, dbj + 2u * kk, kIdescN64, kk > 0 ? 1u : 0u);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) umma_f16(acc, dhi + 2u * kk, dbj + 512u + 2u * kk, kIdescN64, 1u);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) umma_f16(acc, dlo + 2u * kk, dbj + 2u * kk, kIdescN64, 1u);
        umma_commit(my_mbar);
      }
      if (et < 32) {
        // one warp polls the mbarrier; the engine's other warps wait at the
        // named barrier below without taking issue slots
        uint32_t it = 0;
        bool done = false;
        const uint32_t wait_bar = inject ? never_s : my_mbar;
        while (!(done = mbar_try_wait(wait_bar, inject ? 0u : phase)) && ++it < first_limit) {
        }
        if (!done) {
          atomicExch(err, 1);
          s_abort[e] = 1;
          // the MMAs may still be running: one more bounded wait (of the
          // default length, whatever the first wait's limit) before this
          // engine stops and the CTA's normal exit frees the accumulators
          for (uint32_t w = 0; w < 4 * kTcWaitLimit && !mbar_try_wait(my_mbar, phase); ++w) {
          }
        }
        tc_fence_before();
      }
      {
        engine_sync(e);
        phase ^= 1u;
        if (s_abort[e]) {
          aborted = true;
          break;
        }
      }
      tc_fence_after();
      // ---- epilogue of unitary j ----
      const bool last = j + 1 == m;
      // the last MMAs are done, so the operand buffer is free: the next tile's
      // copies fly while this tile's epilogue stores to HBM
      if (last && tile + stride < n_tiles) issue_loads(tile + stride);
      uint32_t my_ptn = 0;
      bool my_pair = false;
#pragma unroll
      for (int jj = 0; jj < kTcMaxUnitaries; ++jj)
        if (jj == j) {
          my_ptn = ptn[jj];
          my_pair = pair[jj];
        }
      // column c = kTcCols ch + 4 part + cc (+ 1 for the second amplitude of
      // a pair): its offsets are the XOR (operand) / sum (amplitude) of one
      // table entry per set bit
      float2 nout = make_float2(0.0f, 0.0f);
      // the mid epilogues need only the operand offsets, the last one only
      // the amplitude offsets: two compile-time forms of the drain loop
      auto drain = [&](auto last_c, auto wide_c) {
        constexpr bool kLast = decltype(last_c)::value;
        // kWide: 8-byte operand stores of column pairs (mid) / 16-byte HBM
        // stores of amplitude pairs (last)
        constexpr bool kWide = decltype(wide_c)::value;
        uint32_t xb[5];
        uint64_t gb[5];
#pragma unroll
        for (int i = 0; i < 5; ++i) {
          if constexpr (kLast) gb[i] = T->gcb[j][i];
          else xb[i] = T->xcb[j][i];
        }
        uint32_t xbase = my_ptn;
        uint64_t gbase = tb + pg;
        if (kTcColHalves == 2 && ch) {
          if constexpr (kLast) gbase += gb[4];
          else xbase ^= xb[4];
        }
        float2* out = reinterpret_cast<float2*>(amp) + gbase;
        const float scv = kLast ? out_scale : mid_scale;
        const float2 sc = make_float2(scv, scv);
#pragma unroll
        for (int pb = 0; pb < kTcParts; pb += kTcBatch) {
          uint32_t rh[kTcBatch][8];
#pragma unroll
          for (int k = 0; k < kTcBatch; ++k) tmem_ld8(lanes + 8u * uint32_t(pb + k), rh[k]);
          tmem_ld_wait();
          if constexpr (kLast) {
            // low index bits onto lanes: whole 128-byte lines per warp store
            // (the exchanges are read from the shared pass record here, so no
            // register holds them across the drain)
            const int s0 = P.sw_lane[0], s1 = P.sw_lane[1], s2 = P.sw_lane[2];
            if (s0 >= 0) lane_swap<1>(rh, 1u << s0, (lane >> s0) & 1);
            if constexpr (kTcMaxLaneSwaps >= 2)
              if (s1 >= 0) lane_swap<2>(rh, 1u << s1, (lane >> s1) & 1);
            if constexpr (kTcMaxLaneSwaps >= 3)
              if (s2 >= 0) lane_swap<3>(rh, 1u << s2, (lane >> s2) & 1);
          }
#pragma unroll
          for (int k = 0; k < kTcBatch; ++k) {
#pragma unroll
            for (int cc = 0; cc < 4; cc += 2) {
              const int cb = 4 * (pb + k) + cc;  // column bits below the column half (compile time)
              // out = D * scale, packed (re, im)
              const float2 x0 =
                  __fmul2_rn(make_float2(__uint_as_float(rh[k][2 * cc]), __uint_as_float(rh[k][2 * cc + 1])), sc);
              const float2 x1 =
                  __fmul2_rn(make_float2(__uint_as_float(rh[k][2 * cc + 2]), __uint_as_float(rh[k][2 * cc + 3])), sc);
              if constexpr (!kLast) {
                uint32_t xo = 0;
#pragma unroll
                for (int b = 1; b < 5; ++b)
                  if ((cb >> b) & 1) xo ^= xb[b];
                const uint32_t o0 = xbase ^ xo;
                if constexpr (kWide) {
                  put2(o0, x0, x1);
                } else {
                  put1(o0, x0);
                  put1(o0 ^ xb[0], x1);
                }
              } else {
                uint64_t go = 0;
#pragma unroll
                for (int b = 1; b < 5; ++b)
                  if ((cb >> b) & 1) go += gb[b];
                nout = __ffma2_rn(x1, x1, __ffma2_rn(x0, x0, nout));
                float2* o0 = out + go;
                if constexpr (kWide) {
                  __stcs(reinterpret_cast<float4*>(o0), make_float4(x0.x, x0.y, x1.x, x1.y));
                } else {
                  __stcs(o0, x0);
                  __stcs(o0 + gb[0], x1);
                }
              }
            }
          }
        }
      };
      // (measured on the 30-qubit brickwork: compile-time pairing forms here
      // and in the split above together +1.5 %, here alone -1.5 %, in the
      // split alone -1 % with a 16-byte spill: code layout, not arithmetic)
      if (last) {
        if (store16) drain(std::true_type{}, std::true_type{});
        else drain(std::true_type{}, std::false_type{});
      } else {
        if (my_pair) drain(std::false_type{}, std::true_type{});
        else drain(std::false_type{}, std::false_type{});
      }
      if (last) norm_out += double(nout.x) + double(nout.y);
      else fence_proxy_async_smem();
      engine_barrier();  // the accumulator is drained before the next MMAs overwrite it
    }
    if (aborted) break;
  }

  cp_async_wait0();  // no copy outlives the CTA (an aborted engine may leave one in flight)

  // ---- per-CTA FP64 norm partials (fixed-order reduction), teardown ----
  tc_fence_before();
  double a = norm_out, b = norm_in;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    s_red[0][warp] = a;
    s_red[1][warp] = b;
  }
  __syncthreads();
  tc_fence_after();
  if (tid == 0) {
    double ta = 0.0, tb2 = 0.0;
    for (int w = 0; w < kTcThreads / 32; ++w) {
      ta += s_red[0][w];
      tb2 += s_red[1][w];
    }
    out_norm[blockIdx.x] = ta;
    if (norm0_out) norm0_out[blockIdx.x] = tb2;
  }
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTcTmemCols));
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct TcPlanImpl {
  TcPlan plan;
  std::vector<size_t> bmat_off;   // first B-operand half of each pass
  TcPassRec* d_passes = nullptr;
  uint16_t* d_bmats = nullptr;
};

bool tc_plan_build(const std::vector<Op>& ops, int n, DType dt, void** plan, PlanStats* stats) {
  *plan = nullptr;
  if (dt != DType::C64) return false;
  auto* p = new TcPlanImpl();
  std::string err;
  if (!build_tc_plan(ops, n, &p->plan, &err)) {
    delete p;
    return false;
  }
  size_t off = 0;
  for (const TcPassRec& P : p->plan.passes) {
    p->bmat_off.push_back(off);
    off += size_t(P.m) * kTcBmatHalves;
  }
  const size_t np = std::max<size_t>(1, p->plan.passes.size());
  bool ok = cudaMalloc(reinterpret_cast<void**>(&p->d_passes), np * sizeof(TcPassRec)) == cudaSuccess;
  ok = ok && cudaMalloc(reinterpret_cast<void**>(&p->d_bmats), std::max<size_t>(8, off) * sizeof(uint16_t)) ==
                 cudaSuccess;
  if (ok && !p->plan.passes.empty())
    ok = cudaMemcpy(p->d_passes, p->plan.passes.data(), p->plan.passes.size() * sizeof(TcPassRec),
                    cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok && off)
    ok = cudaMemcpy(p->d_bmats, p->plan.bmats.data(), off * sizeof(uint16_t), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    tc_plan_free(p);
    return false;
  }
  *stats = p->plan.stats;
  *plan = p;
  return true;
}

bool tc_plan_stats(const std::vector<Op>& ops, int n, DType dt, PlanStats* stats) {
  if (dt != DType::C64) return false;
  TcPlan tp;
  std::string err;
  if (!build_tc_plan(ops, n, &tp, &err, false)) return false;
  *stats = tp.stats;
  return true;
}

void tc_plan_free(void* plan) {
  auto* p = static_cast<TcPlanImpl*>(plan);
  if (!p) return;
  if (p->d_passes) cudaFree(p->d_passes);
  if (p->d_bmats) cudaFree(p->d_bmats);
  delete p;
}

// Polls of an engine's first wait for its MMAs before it gives up (sets the
// error flag, then waits up to 4 x the default for the MMAs in flight, so
// that no MMA outlives the CTA's tensor memory).  Bit 31 makes that first
// wait poll a barrier nothing arrives on, so it expires: the failure
// injection of nqpu_tensor_wait_limit_set.
std::atomic<uint32_t> g_tc_wait_limit{kTcWaitLimit};

cudaError_t tc_launch(float* amp, const TcPlan& plan, const TcPassRec* d_passes, const uint16_t* d_bmats,
                      const size_t* bmat_off, double* d_norm, int slots, int* d_err, cudaStream_t st,
                      std::vector<cudaEvent_t>* events) {
  static PerDeviceOnce<cudaError_t> attr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = attr.get(dev, [] { return cudaFuncSetAttribute(k_tc_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTcSmem)); },
               cudaErrorInvalidDevice);
  if (e != cudaSuccess) return e;
  // the expiry flag of an earlier run is cleared, so this run reports its own
  if ((e = cudaMemsetAsync(d_err, 0, sizeof(int), st)) != cudaSuccess) return e;
  const uint32_t wait_limit = g_tc_wait_limit.load(std::memory_order_relaxed);
  const uint32_t n_tiles = uint32_t(1) << (plan.n - kTcTileBits);
  const unsigned grid =
      unsigned(std::min<uint64_t>((uint64_t(n_tiles) + kTcEngines - 1) / kTcEngines, uint64_t(slots)));
  double* norm0 = d_norm;
  for (size_t i = 0; i < plan.passes.size(); ++i) {
    double* outn = d_norm + (1 + (i & 1)) * size_t(slots);
    const double* prevn = i ? d_norm + (1 + ((i + 1) & 1)) * size_t(slots) : nullptr;
    k_tc_pass<<<grid, kTcThreads, kTcSmem, st>>>(amp, d_passes + i, d_bmats + bmat_off[i], n_tiles, plan.state_scale,
                                                  i ? norm0 : nullptr, i ? nullptr : norm0, prevn, int(grid), outn,
                                                  d_err, wait_limit);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (events) {
      cudaEvent_t ev;
      if ((e = cudaEventCreate(&ev)) != cudaSuccess) return e;
      events->push_back(ev);
      if ((e = cudaEventRecord(ev, st)) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

void tc_bmat_offsets(const TcPlan& plan, std::vector<size_t>* off) {
  off->clear();
  size_t o = 0;
  for (const TcPassRec& P : plan.passes) {
    off->push_back(o);
    o += size_t(P.m) * kTcBmatHalves;
  }
}

cudaError_t tc_run(void* plan, StateImpl* s, std::vector<cudaEvent_t>* events) {
  auto* p = static_cast<TcPlanImpl*>(plan);
  if (!p || s->dt != DType::C64 || int(s->n) != p->plan.n) return cudaErrorInvalidValue;
  // norm partials ([norm0 | out ping | out pong], one slot per CTA) and the
  // expiry flag of this run: the state's scratch
  const int slots = device_sms();
  double* norm = nullptr;
  int* err = nullptr;
  const cudaError_t e = state_run_scratch(s, 3 * size_t(slots), &norm, &err);
  if (e != cudaSuccess) return e;
  return tc_launch(static_cast<float*>(s->amp), p->plan, p->d_passes, p->d_bmats, p->bmat_off.data(), norm, slots,
                   err, s->stream, events);
}


}  // namespace nqpu

// Diagnostics: the tensor passes' first MMA wait (0 polls = the default).
extern "C" NqpuError nqpu_tensor_wait_limit_set(uint32_t polls, int32_t never_arrives) {
  if (polls > 0x7FFFFFFFu) return NQPU_INVALID_PARAMETER;
  const uint32_t v = (polls ? polls : nqpu::kTcWaitLimit) | (never_arrives ? 0x80000000u : 0u);
  nqpu::g_tc_wait_limit.store(v, std::memory_order_relaxed);
  return NQPU_OK;
}
