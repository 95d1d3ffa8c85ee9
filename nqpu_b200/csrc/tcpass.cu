// Tensor-core pass mode (complex64): several fused 5-qubit unitaries per HBM
// pass, each applied as a split-TF32 tcgen05 GEMM on a tile held in shared
// memory (plan data and layouts in tcpass.h, planner in tcplan.cpp).
//
// Per pass, one persistent CTA per SM with two independent tile engines
// ("groups" of sixteen warps).  A group owns an operand buffer (the tile as the
// 128 x 64 fp32 A operand, hi and lo TF32 planes, K-major 128-byte swizzle) and
// a 128-column TMEM accumulator, and runs its tiles through:
//   load     4 coalesced 16-byte HBM loads per thread (a tile = 128 runs of
//            32 amplitudes), scale by the renormalisation factor, split into
//            TF32 hi/lo and store into the operand in unitary 0's layout;
//   unitary  one elected thread issues 16 MMAs: D[:, 0:128] = A_hi [R_hi; R_lo]^T
//            (N = 128, K = 64) then D[:, 0:64] += A_lo R_hi^T (N = 64), and
//            commits them to the group's mbarrier (bounded wait);
//   epilogue each thread reads a quarter of its row (TMEM lane) of D: warps
//            w, w + 4, w + 8, w + 12 of a group share a lane quadrant and take
//            8 columns each; it adds the two halves of D (out = A_hi R_hi +
//            A_lo R_hi + A_hi R_lo) and either splits its 8 amplitudes straight
//            into the next unitary's operand layout, or, after the last
//            unitary, stores them to HBM.
// While one group waits for its MMAs the other runs its loads and epilogues,
// so the tensor pipe, shared memory and HBM overlap across the two tiles.
// The B operands of the pass's unitaries stay in shared memory for the launch.
//
// Renormalisation: the first pass of a run records the FP64 norm of its input
// (per-CTA partials) and every pass the norm of its output; each later pass
// scales its input by sqrt(norm_in / norm_prev_out), so the norm drift of the
// TF32 contractions is removed without an extra HBM pass and the state keeps
// the norm it had when the run started.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_once.h"
#include "engine.h"
#include "kernels.h"
#include "tcpass.h"
#include "tcrun.h"
#include "umma.cuh"

namespace nqpu {

constexpr int kTcThreads = 1024;
constexpr int kTcGroupThreads = 512;
constexpr int kTcLoadSteps = 4;  // 16-byte loads per thread per tile
constexpr uint32_t kTcAPlane = 128 * 64 * 4;         // 32 KB: 128 rows x 64 fp32
constexpr uint32_t kTcOpBytes = 2 * kTcAPlane;       // hi + lo planes
constexpr uint32_t kTcBBytes = 128 * 64 * 4;         // [R_hi; R_lo]: 128 rows x 64 fp32
constexpr uint32_t kTcAtom = 128 * 128;              // one K-atom (32 fp32) of 128 rows
constexpr uint32_t kTcWaitLimit = 1u << 22;          // bounded mbarrier polls
constexpr uint32_t kTcTmemCols = 512;                // two groups x two 128-column accumulators
static_assert(kTcThreads == 2 * kTcGroupThreads, "two tile engines per CTA");

struct TcTables {
  uint32_t xnext[kTcMaxUnitaries][32];
  uint64_t gcol[kTcMaxUnitaries][32];
  uint32_t sol[kTcLoadSteps];  // loader: operand offset (unitary 0's layout) of load step i
  uint64_t sgl[kTcLoadSteps];  // loader: amplitude offset of load step i
};

constexpr size_t kTcSmem = 1024 /*alignment*/ + 2 * size_t(kTcOpBytes) + kTcMaxUnitaries * size_t(kTcBBytes) +
                           sizeof(TcTables);
static_assert(kTcSmem <= 232448, "dynamic shared memory of one CTA");

constexpr uint32_t kIdescN128 = umma_idesc_tf32<128, 128>();
constexpr uint32_t kIdescN64 = umma_idesc_tf32<128, 64>();

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(1 + g), "n"(kTcGroupThreads) : "memory");
}

__global__ void __launch_bounds__(kTcThreads, 1)
    k_tc_pass(float* __restrict__ amp, const TcPassRec* __restrict__ pass, const float* __restrict__ bmats,
              uint32_t n_tiles, const double* __restrict__ norm0, double* __restrict__ norm0_out,
              const double* __restrict__ prev_norm, int n_prev, double* __restrict__ out_norm,
              int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw_s = static_cast<uint32_t>(__cvta_generic_to_shared(smem_raw));
  unsigned char* base_p = smem_raw + ((1024 - (raw_s & 1023)) & 1023);
  unsigned char* opbuf = base_p;                            // [2][hi | lo]
  unsigned char* bbuf = base_p + 2 * kTcOpBytes;            // [m][128 rows x 64 fp32]
  TcTables* T = reinterpret_cast<TcTables*>(bbuf + kTcMaxUnitaries * kTcBBytes);
  __shared__ TcPassRec P;
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_holder;
  __shared__ int s_abort[2];
  __shared__ double s_red[2][kTcThreads / 32];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = tid >> 9, gt = tid & (kTcGroupThreads - 1);
  const int q = warp & 3, cq = (warp >> 2) & 3;  // TMEM lane quadrant, column quarter
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
    const float4* bsrc = reinterpret_cast<const float4*>(bmats + size_t(j) * kTcBmatFloats);
    unsigned char* bdst = bbuf + j * kTcBBytes;
    for (int e = tid; e < int(kTcBmatFloats / 4); e += kTcThreads) {
      const uint32_t nrow = uint32_t(e) >> 4, k = (uint32_t(e) & 15u) * 4u;
      *reinterpret_cast<float4*>(bdst + tc_sw128_off<128>(nrow, k)) = __ldg(bsrc + e);
    }
  }
  for (int i = tid; i < m * 32; i += kTcThreads) {
    T->xnext[i >> 5][i & 31] = P.u[i >> 5].xnext[i & 31];
    T->gcol[i >> 5][i & 31] = P.u[i >> 5].gcol[i & 31];
  }
  if (tid < kTcLoadSteps) {
    uint32_t o = 0;
    uint64_t a = 0;
    for (int s = 0; s < 2; ++s)
      if ((tid >> s) & 1) {
        o ^= P.u[0].boff[P.lt[9 + s]];
        a |= 1ull << P.qt[P.lt[9 + s]];
      }
    T->sol[tid] = o;
    T->sgl[tid] = a;
  }
  const uint32_t mbar_s = static_cast<uint32_t>(__cvta_generic_to_shared(&mbar[0]));
  if (tid == 0) {
    mbar_init(mbar_s, 1);
    mbar_init(mbar_s + 8, 1);
    s_abort[0] = s_abort[1] = 0;
  }
  if (warp == 0) {
    const uint32_t holder = static_cast<uint32_t>(__cvta_generic_to_shared(&tmem_holder));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(holder),
                 "r"(kTcTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  fence_proxy_async_smem();  // the B operands, written by generic stores, are read by the tensor core
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_holder;

  // renormalisation factor of this pass's input
  float scale = 1.0f;
  if (prev_norm && norm0) {
    double t0 = 0.0, tp = 0.0;
    for (int i = 0; i < n_prev; ++i) {
      t0 += norm0[i];
      tp += prev_norm[i];
    }
    if (t0 > 0.0 && tp > 0.0) scale = float(sqrt(t0 / tp));
  }

  // ---- per-thread address parts ----
  // loader: thread bit b of gt is tile bit lt[b], step bit s is tile bit
  // lt[9 + s], and tile bit 0 is the pair inside each 16-byte load
  uint32_t pol = 0;
  uint64_t pgl = 0;
  for (int b = 0; b < 9; ++b)
    if ((gt >> b) & 1) {
      pol ^= P.u[0].boff[P.lt[b]];
      pgl |= 1ull << P.qt[P.lt[b]];
    }
  const uint32_t boff_h = P.u[0].boff[0];
  const bool load16 = boff_h == 8u;  // tile bit 0 is column bit 0: (h = 0, 1) share a 16-byte chunk
  // epilogue of unitary j: row part of the thread's row (its TMEM lane)
  uint32_t ptn[kTcMaxUnitaries];
  bool pair16[kTcMaxUnitaries];
  uint64_t pg = 0;
#pragma unroll
  for (int j = 0; j < kTcMaxUnitaries; ++j) {
    ptn[j] = 0;
    pair16[j] = false;
    if (j + 1 < m) {
      for (int i = 0; i < 7; ++i)
        if ((row >> i) & 1u) ptn[j] ^= P.u[j + 1].boff[P.u[j].frow[i]];
      pair16[j] = P.u[j + 1].boff[P.u[j].fcol[0]] == 8u;
    } else if (j + 1 == m) {
      for (int i = 0; i < 7; ++i)
        if ((row >> i) & 1u) pg |= 1ull << P.qt[P.u[j].frow[i]];
    }
  }
  const bool store16 = P.qt[P.u[m - 1].fcol[0]] == 0;  // qubit 0 is column bit 0 of the last layout

  const uint32_t ahi_s = static_cast<uint32_t>(__cvta_generic_to_shared(opbuf)) + uint32_t(g) * kTcOpBytes;
  const uint32_t alo_s = ahi_s + kTcAPlane;
  const uint32_t b_s = static_cast<uint32_t>(__cvta_generic_to_shared(bbuf));
  const uint32_t my_mbar = mbar_s + 8u * uint32_t(g);

  // split (re, im) pairs into the hi and lo operand planes at byte offset o
  auto put2 = [&](uint32_t o, float re, float im) {
    const float hr = tf32_rn(re), hi = tf32_rn(im);
    sts_v2(ahi_s + o, hr, hi);
    sts_v2(alo_s + o, tf32_rn(re - hr), tf32_rn(im - hi));
  };
  auto put4 = [&](uint32_t o, float4 x) {
    const float4 h = make_float4(tf32_rn(x.x), tf32_rn(x.y), tf32_rn(x.z), tf32_rn(x.w));
    sts_v4(ahi_s + o, h.x, h.y, h.z, h.w);
    sts_v4(alo_s + o, tf32_rn(x.x - h.x), tf32_rn(x.y - h.y), tf32_rn(x.z - h.z), tf32_rn(x.w - h.w));
  };
  auto tile_base_of = [&](uint32_t tile) {
    const uint64_t mine = (lane < P.n_out && ((tile >> lane) & 1u)) ? (1ull << P.qout[lane]) : 0ull;
    const uint32_t lo = __reduce_or_sync(0xffffffffu, uint32_t(mine));
    const uint32_t hi = __reduce_or_sync(0xffffffffu, uint32_t(mine >> 32));
    return uint64_t(lo) | (uint64_t(hi) << 32);
  };

  double norm_in = 0.0, norm_out = 0.0;
  uint32_t phase = 0;   // parity of the group's mbarrier phase to wait for
  uint32_t batches = 0; // MMA batches issued by this group (accumulator = batches & 1)
  const uint32_t stride = 2u * gridDim.x;

  // HBM -> registers (16-byte loads; tile bit 0 is the pair inside each)
  auto load_tile = [&](uint64_t tb, float4 (&v)[kTcLoadSteps]) {
    const float4* src = reinterpret_cast<const float4*>(amp) + ((tb + pgl) >> 1);
#pragma unroll
    for (int i = 0; i < kTcLoadSteps; ++i) v[i] = __ldcs(src + (T->sgl[i] >> 1));
  };
  // registers -> unitary 0's operand: renormalise, split, store
  auto split_tile = [&](const float4 (&v)[kTcLoadSteps]) {
    float tile_in = 0.0f;  // this thread's 8 amplitudes: an FP32 partial, then FP64 across tiles
#pragma unroll
    for (int i = 0; i < kTcLoadSteps; ++i) {
      float4 x = v[i];
      if (norm0_out) tile_in += x.x * x.x + x.y * x.y + x.z * x.z + x.w * x.w;
      x.x *= scale;
      x.y *= scale;
      x.z *= scale;
      x.w *= scale;
      const uint32_t o = pol ^ T->sol[i];
      if (load16) {
        put4(o, x);
      } else {
        put2(o, x.x, x.y);
        put2(o ^ boff_h, x.z, x.w);
      }
    }
    if (norm0_out) norm_in += double(tile_in);
    fence_proxy_async_smem();
  };
  // one elected thread: unitary j's 16 MMAs into the next free accumulator.
  // The descriptors differ only in their start-address field (address >> 4,
  // bits 0..13, which no offset here carries out of), so each is a base
  // descriptor plus a compile-time constant.
  auto issue_unitary = [&](int j) -> uint32_t {
    const uint32_t acc = tmem + 256u * uint32_t(g) + 128u * (batches & 1u);
    if (gt == 0) {
      const uint64_t dhi = umma_desc_sw128(ahi_s), dlo = umma_desc_sw128(alo_s);
      const uint64_t dbj = umma_desc_sw128(b_s + uint32_t(j) * kTcBBytes);
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) {
        const uint64_t off = (uint64_t(kk >> 2) * kTcAtom + uint64_t(kk & 3) * 32u) >> 4;
        umma_tf32(acc, dhi + off, dbj + off, kIdescN128, kk > 0 ? 1u : 0u);
      }
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) {
        const uint64_t off = (uint64_t(kk >> 2) * kTcAtom + uint64_t(kk & 3) * 32u) >> 4;
        umma_tf32(acc, dlo + off, dbj + off, kIdescN64, 1u);
      }
      umma_commit(my_mbar);
    }
    ++batches;
    return acc;
  };
  auto group_barrier = [&]() {
    tc_fence_before();
    group_sync(g);
    tc_fence_after();
  };
  // bounded wait for the group's outstanding MMA batch; false: give up
  auto wait_unitary = [&]() -> bool {
    uint32_t it = 0;
    bool done = false;
    while (!(done = mbar_try_wait(my_mbar, phase)) && ++it < kTcWaitLimit) {
    }
    if (!done) {
      atomicExch(err, 1);
      s_abort[g] = 1;
      // the MMAs may still be running: one more bounded wait before this
      // group stops and the CTA's normal exit frees the accumulators
      for (uint32_t w = 0; w < 4 * kTcWaitLimit && !mbar_try_wait(my_mbar, phase); ++w) {
      }
    }
    group_sync(g);
    phase ^= 1u;
    tc_fence_after();
    return s_abort[g] == 0;
  };
  // epilogue of unitary j (not the last): accumulator -> next operand layout
  auto epilogue_mid = [&](int j, uint32_t acc) {
    uint32_t my_ptn = 0;
    bool my_pair = false;
#pragma unroll
    for (int jj = 0; jj < kTcMaxUnitaries; ++jj)
      if (jj == j) {
        my_ptn = ptn[jj];
        my_pair = pair16[jj];
      }
    const uint32_t lanes = acc + (uint32_t(q * 32) << 16) + 16u * uint32_t(cq);
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      uint32_t rh[8], rl[8];
      tmem_ld8(lanes + 8u * uint32_t(part), rh);
      tmem_ld8(lanes + 64u + 8u * uint32_t(part), rl);
      tmem_ld_wait();
#pragma unroll
      for (int cc = 0; cc < 4; cc += 2) {
        const int c = 8 * cq + 4 * part + cc;
        const float re0 = __uint_as_float(rh[2 * cc]) + __uint_as_float(rl[2 * cc]);
        const float im0 = __uint_as_float(rh[2 * cc + 1]) + __uint_as_float(rl[2 * cc + 1]);
        const float re1 = __uint_as_float(rh[2 * cc + 2]) + __uint_as_float(rl[2 * cc + 2]);
        const float im1 = __uint_as_float(rh[2 * cc + 3]) + __uint_as_float(rl[2 * cc + 3]);
        const uint32_t o0 = my_ptn ^ T->xnext[j][c];
        if (my_pair) {
          put4(o0, make_float4(re0, im0, re1, im1));
        } else {
          put2(o0, re0, im0);
          put2(my_ptn ^ T->xnext[j][c + 1], re1, im1);
        }
      }
    }
    fence_proxy_async_smem();
  };
  // epilogue of the last unitary: accumulator -> HBM, FP64 norm of the output
  auto epilogue_last = [&](uint64_t tb, uint32_t acc) {
    const int j = m - 1;
    const uint32_t lanes = acc + (uint32_t(q * 32) << 16) + 16u * uint32_t(cq);
    float2* out = reinterpret_cast<float2*>(amp) + (tb + pg);
    float tile_out = 0.0f;  // FP32 partial over this thread's 8 amplitudes
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      uint32_t rh[8], rl[8];
      tmem_ld8(lanes + 8u * uint32_t(part), rh);
      tmem_ld8(lanes + 64u + 8u * uint32_t(part), rl);
      tmem_ld_wait();
#pragma unroll
      for (int cc = 0; cc < 4; cc += 2) {
        const int c = 8 * cq + 4 * part + cc;
        const float re0 = __uint_as_float(rh[2 * cc]) + __uint_as_float(rl[2 * cc]);
        const float im0 = __uint_as_float(rh[2 * cc + 1]) + __uint_as_float(rl[2 * cc + 1]);
        const float re1 = __uint_as_float(rh[2 * cc + 2]) + __uint_as_float(rl[2 * cc + 2]);
        const float im1 = __uint_as_float(rh[2 * cc + 3]) + __uint_as_float(rl[2 * cc + 3]);
        tile_out += re0 * re0 + im0 * im0 + re1 * re1 + im1 * im1;
        if (store16) {
          __stcs(reinterpret_cast<float4*>(out + T->gcol[j][c]), make_float4(re0, im0, re1, im1));
        } else {
          __stcs(out + T->gcol[j][c], make_float2(re0, im0));
          __stcs(out + T->gcol[j][c + 1], make_float2(re1, im1));
        }
      }
    }
    norm_out += double(tile_out);
  };

  // Software pipeline over the group's tiles t0, t1, ...: the HBM loads of
  // tile t+1 are issued as tile t's first MMAs start and land in registers
  // while tile t runs (no further prefetch: more loads in flight only throttle
  // the load-store unit); when tile t's last MMAs are done the operand buffer is
  // free, so tile t+1 is split into it and its first MMAs run (into the other
  // accumulator) while tile t's last epilogue drains to HBM.
  uint32_t tile = 2u * blockIdx.x + uint32_t(g);
  if (tile < n_tiles) {
    float4 v[kTcLoadSteps];
    uint64_t tb = tile_base_of(tile);
    load_tile(tb, v);
    split_tile(v);
    group_barrier();
    uint32_t acc = issue_unitary(0);
    for (;;) {
      const uint32_t next = tile + stride;
      const bool has_next = next < n_tiles;
      uint64_t ntb = 0;
      if (has_next) {
        ntb = tile_base_of(next);
        load_tile(ntb, v);  // registers free since the split of `tile`
      }
      bool ok = true;
      for (int j = 0; j < m && ok; ++j) {
        ok = wait_unitary();
        if (!ok) break;
        if (j + 1 < m) {
          epilogue_mid(j, acc);  // writes the operand the finished MMAs read
          group_barrier();
          acc = issue_unitary(j + 1);
        } else {
          const uint32_t acc_last = acc;
          if (has_next) {
            split_tile(v);  // the operand is free: tile `next` goes in
            group_barrier();
            acc = issue_unitary(0);  // into the other accumulator
          }
          epilogue_last(tb, acc_last);
          group_barrier();  // acc_last drained before an MMA reuses it
        }
      }
      if (!ok || !has_next) break;
      tile = next;
      tb = ntb;
    }
  }

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
  std::vector<size_t> bmat_off;   // first B-operand float of each pass
  TcPassRec* d_passes = nullptr;
  float* d_bmats = nullptr;
  double* d_norm = nullptr;       // [norm0 | out ping | out pong], `slots` doubles each
  int slots = 0;
  int* d_err = nullptr;
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
    off += size_t(P.m) * kTcBmatFloats;
  }
  const size_t np = std::max<size_t>(1, p->plan.passes.size());
  bool ok = cudaMalloc(reinterpret_cast<void**>(&p->d_passes), np * sizeof(TcPassRec)) == cudaSuccess;
  ok = ok && cudaMalloc(reinterpret_cast<void**>(&p->d_bmats), std::max<size_t>(1, off) * sizeof(float)) == cudaSuccess;
  if (ok && !p->plan.passes.empty())
    ok = cudaMemcpy(p->d_passes, p->plan.passes.data(), p->plan.passes.size() * sizeof(TcPassRec),
                    cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok && off)
    ok = cudaMemcpy(p->d_bmats, p->plan.bmats.data(), off * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
  p->slots = device_sms();
  ok = ok && cudaMalloc(reinterpret_cast<void**>(&p->d_norm), sizeof(double) * 3 * size_t(p->slots)) == cudaSuccess;
  ok = ok && cudaMalloc(reinterpret_cast<void**>(&p->d_err), sizeof(int)) == cudaSuccess;
  ok = ok && cudaMemset(p->d_err, 0, sizeof(int)) == cudaSuccess;
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
  if (!build_tc_plan(ops, n, &tp, &err)) return false;
  *stats = tp.stats;
  return true;
}

void tc_plan_free(void* plan) {
  auto* p = static_cast<TcPlanImpl*>(plan);
  if (!p) return;
  if (p->d_passes) cudaFree(p->d_passes);
  if (p->d_bmats) cudaFree(p->d_bmats);
  if (p->d_norm) cudaFree(p->d_norm);
  if (p->d_err) cudaFree(p->d_err);
  delete p;
}

cudaError_t tc_run(void* plan, StateImpl* s, std::vector<cudaEvent_t>* events) {
  auto* p = static_cast<TcPlanImpl*>(plan);
  if (!p || s->dt != DType::C64 || int(s->n) != p->plan.n) return cudaErrorInvalidValue;
  static PerDeviceOnce<cudaError_t> attr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = attr.get(dev, [] { return cudaFuncSetAttribute(k_tc_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTcSmem)); },
               cudaErrorInvalidDevice);
  if (e != cudaSuccess) return e;
  const uint64_t n_tiles = 1ull << (p->plan.n - kTcTileBits);
  const unsigned grid = unsigned(std::min<uint64_t>((n_tiles + 1) / 2, uint64_t(p->slots)));
  double* norm0 = p->d_norm;
  for (size_t i = 0; i < p->plan.passes.size(); ++i) {
    double* outn = p->d_norm + (1 + (i & 1)) * size_t(p->slots);
    const double* prevn = i ? p->d_norm + (1 + ((i + 1) & 1)) * size_t(p->slots) : nullptr;
    k_tc_pass<<<grid, kTcThreads, kTcSmem, s->stream>>>(
        static_cast<float*>(s->amp), p->d_passes + i, p->d_bmats + p->bmat_off[i], uint32_t(n_tiles), i ? norm0 : nullptr,
        i ? nullptr : norm0, prevn, int(grid), outn, p->d_err);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (events) {
      cudaEvent_t ev;
      if ((e = cudaEventCreate(&ev)) != cudaSuccess) return e;
      events->push_back(ev);
      if ((e = cudaEventRecord(ev, s->stream)) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

cudaError_t tc_check_error(void* plan, cudaStream_t st) {
  auto* p = static_cast<TcPlanImpl*>(plan);
  if (!p) return cudaSuccess;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  return h ? cudaErrorLaunchTimeout : cudaSuccess;
}

}  // namespace nqpu
