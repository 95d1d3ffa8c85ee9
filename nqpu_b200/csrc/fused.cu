// Fused execution mode (precision form).
//
// Host: a fusion pass packs runs of gates into dense <=5-qubit unitaries.  It
// generalises the reference's fuse_gates (circuits/synthesis/gate_fusion.rs:537:
// 1q runs -> 2x2, absorption into 2q gates -> 4x4) from 2 to 5 qubits: ops are
// taken greedily in circuit order while the union of their qubits stays within
// 5, and an op may move ahead of a deferred op only when they share no qubit.
// Each cluster's 32x32 unitary is accumulated in FP64 by applying the cluster's
// ops to the 32 basis columns.
//
// Device: one launch per fused unitary U on qubits F = (f0 < ... < f4).  The
// state is viewed as groups of 32 amplitudes (the F-subspace of a fixed
// assignment of the other qubits).  A CTA takes 128 groups at a time and
// computes out_g = U v_g for all of them as one tensor-core GEMM on the real
// embedding:  D[128 x 64] = A[128 x 64] * B^T, A row g = (re, im) of the 32
// amplitudes of group g, B = R (64 x 64 real form of U).  Inputs are split
// into TF32 hi/lo parts (hi = x rounded to TF32, lo = the remainder rounded to
// TF32) and D = A_hi B_hi + A_hi B_lo + A_lo B_hi is accumulated in FP32 in
// tensor memory by tcgen05.mma kind::tf32 (24 MMAs of 128x64x8 per tile).
// Operands live in shared memory in the K-major 128-byte-swizzled layout.
//
// HBM access: a tile's 4096 amplitudes form a 12-dimensional sub-cube (F and
// the 7 lowest qubits outside F, which always include qubits 0..6).  Loads
// walk the sub-cube in its own linear order, so each warp moves 512 contiguous
// bytes per 16-byte instruction; the (row, column) of every amplitude in A
// follows from the same bits.  Results go from tensor memory straight to HBM:
// a warp's lanes hold 32 rows of D, whose low row bits the group-row order
// gives to the unfused qubits among 0..4, so that the stores stay coalesced
// (32 neighbouring amplitudes when none of qubits 0..4 is fused).  Two CTAs
// of eight warps share an SM, so one CTA's HBM traffic overlaps the other's
// MMAs, and four warps per scheduler hide the latencies of the operand split
// and the epilogue.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "device_once.h"
#include "engine.h"
#include "fused.h"
#include "fusion.h"
#include "kernels.h"
#include "sv_device.cuh"
#include "umma.cuh"

namespace nqpu {

// ---------------------------------------------------------------------------
// Device kernel
// ---------------------------------------------------------------------------
// Eight warps with two roles: warps 0-3 load tiles from HBM and split them
// into the operand planes, warps 4-7 drain the accumulators (one group row
// per thread, TMEM lane = row) to HBM.
constexpr int kFusedThreads = 256;
constexpr int kProdThreads = 128;          // warps 0-3
constexpr int kTidBits = 7;                // log2(kProdThreads)
constexpr int kLoadSteps = 4096 / (2 * kProdThreads);  // 16-byte loads per loading thread per tile
static_assert((1 << kTidBits) == kProdThreads && kLoadSteps == 16, "fused tile decomposition");
constexpr int kAtomBytes = 128 * 128;      // one K-atom (32 tf32) of 128 rows
constexpr int kAPlane = 2 * kAtomBytes;    // 32 KB: 128 rows x 64 tf32
constexpr int kBPlane = 2 * 64 * 128;      // 16 KB: 64 rows x 64 tf32
constexpr int kSmemFused = 2 * kAPlane + 2 * kBPlane + 1024 /*align*/ + 2048 /*tables*/;
constexpr uint32_t kWaitLimit = 1u << 22;  // bounded mbarrier wait (iterations)

struct FusedArgs {
  int n;
  int q[5];               // fused qubits ascending
  int gq[7];              // group bits: the 7 lowest qubits outside F (or fewer when n < 12)
  int ng;                 // number of group bits used
  int n_out;              // tile-id bits
  int qout[kMaxQubits];   // qubits of tile-id bits
  int lane_over_j;        // 1: F contains qubit 0
  int rot;                // 1: load step of lane L is (i + L / 8) % 8 (column bit 0 is a step bit)
  int sub[12];            // sub-cube qubits (sub[0..5] = 0..5)
  int sub_row[12];        // >= 0: row (group) bit of sub-cube bit b, else -1
  int sub_col[12];        // >= 0: column (F) bit of sub-cube bit b, else -1
};

// Byte offset of element (row r, fp32 column k) in a K-major SW128 operand of
// `rows` rows: K-atom (32 fp32 = 128 B per row) stride rows * 128 B, 8-row
// groups at 1024 B, 16-byte chunks XOR-swizzled with the row within the group.
template <uint32_t kRows>
__device__ __forceinline__ uint32_t sw128_off(uint32_t r, uint32_t k) {
  const uint32_t atom = k >> 5;
  const uint32_t byte = (k & 31) * 4;
  const uint32_t chunk = byte >> 4, within = byte & 15;
  return atom * (kRows * 128u) + (r >> 3) * 1024 + (r & 7) * 128 + ((chunk ^ (r & 7)) << 4) + within;
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) { return umma_desc_sw128(saddr); }

// kind::tf32, D fp32, A/B tf32, both K-major, N = 64, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
static_assert(kIdesc == umma_idesc_tf32<128, 64>(), "instruction descriptor");

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// Renormalisation: every launch writes the FP64 sum of |out|^2 of the tiles it
// processed to out_norm[blockIdx.x]; the next launch sums those partials (in a
// fixed order) and scales its own output by 1/sqrt(sum), so the norm drift of
// each fused unitary is removed by the next one at no extra HBM pass.
constexpr int kFusedCtasPerSm = 2;

__global__ void __launch_bounds__(kFusedThreads, kFusedCtasPerSm)
    k_fused_apply(float* __restrict__ amp, FusedArgs A, const float* __restrict__ bmat /* hi[64][64], lo[64][64] */,
                  const double* __restrict__ prev_norm, int n_prev, double* __restrict__ out_norm,
                  uint64_t n_tiles, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-aligned operand region
  const uint32_t raw_s = static_cast<uint32_t>(__cvta_generic_to_shared(smem_raw));
  const uint32_t pad = (1024 - (raw_s & 1023)) & 1023;
  unsigned char* base = smem_raw + pad;
  unsigned char* a_hi = base;
  unsigned char* a_lo = base + kAPlane;
  unsigned char* b_hi = base + 2 * kAPlane;
  unsigned char* b_lo = b_hi + kBPlane;
  uint64_t* it_addr = reinterpret_cast<uint64_t*>(b_lo + kBPlane);  // kLoadSteps entries
  uint32_t* it_op = reinterpret_cast<uint32_t*>(it_addr + 16);        // kLoadSteps entries: operand offset part
  uint64_t* ctab = reinterpret_cast<uint64_t*>(it_op + 16);           // 32 entries: amplitude offset of column j
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_holder;
  __shared__ int abort_flag;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t mbar_addr = static_cast<uint32_t>(__cvta_generic_to_shared(&mbar));

  // Sub-cube index u = h | tid << 1 | i << (1 + kTidBits) (h: amplitude in a
  // 16-byte pair, tid: loading thread, i: load step).  Global offset, row and column of u are XORs of the parts.
  auto part = [&](uint32_t u, uint64_t* addr, uint32_t* row, uint32_t* col) {
    uint64_t a = 0;
    uint32_t r = 0, c = 0;
    for (int b = 0; b < 12; ++b)
      if ((u >> b) & 1u) {
        a |= 1ull << A.sub[b];
        if (A.sub_row[b] >= 0) r |= 1u << A.sub_row[b];
        else c |= 1u << A.sub_col[b];
      }
    *addr = a;
    *row = r;
    *col = c;
  };
  // The swizzled operand offset sw128_off(r, 2c) is GF(2)-linear in the bits
  // of (r, c) (its fields occupy disjoint bits), so the offset of sub-cube
  // index u = h | tid << 1 | step << 8 is the XOR of the offsets of its parts.
  auto op_off = [&](uint32_t r, uint32_t c) { return sw128_off<128>(r, 2 * c); };
  if (tid < kLoadSteps) {
    uint64_t a;
    uint32_t r, c;
    part(uint32_t(tid) << (1 + kTidBits), &a, &r, &c);
    it_addr[tid] = a;
    it_op[tid] = op_off(r, c);
  }
  if (tid < 32) {
    uint64_t o = 0;
    for (int b = 0; b < 5; ++b)
      if ((tid >> b) & 1) o |= 1ull << A.q[b];
    ctab[tid] = o;
  }
  // load-step rotation by lane group (8 lanes = 128 contiguous bytes stay together)
  const uint32_t g = A.rot ? uint32_t((lane >> 3) & 3) : 0u;
  const bool loader = tid < kProdThreads;
  uint64_t t_addr;
  uint32_t t_row, t_col, h_row, h_col;
  {
    uint64_t a;
    part(uint32_t(tid & (kProdThreads - 1)) << 1, &t_addr, &t_row, &t_col);
    part(1u, &a, &h_row, &h_col);
  }
  const uint32_t op_t = op_off(t_row, t_col), op_h = op_off(h_row, h_col);
  // amplitude offset of this thread's output row (row = tid % 128: its TMEM lane)
  uint64_t row_addr = 0;
  for (int b = 0; b < 12; ++b)
    if (A.sub_row[b] >= 0 && ((uint32_t(tid & 127) >> A.sub_row[b]) & 1u)) row_addr |= 1ull << A.sub[b];
  // qubit of tile-id bit `lane` (tile bases are built by a warp-wide OR)
  const uint64_t lane_bit = lane < A.n_out ? (1ull << A.qout[lane]) : 0ull;
  // B operand (constant for the launch): row n (output real index), col k
  for (int i = tid; i < 64 * 64; i += blockDim.x) {
    const uint32_t r = i >> 6, k = i & 63;
    *reinterpret_cast<float*>(b_hi + sw128_off<64>(r, k)) = __ldg(bmat + i);
    *reinterpret_cast<float*>(b_lo + sw128_off<64>(r, k)) = __ldg(bmat + 4096 + i);
  }
  if (tid == 0) {
    mbar_init(mbar_addr, 1);
    abort_flag = 0;
  }
  if (warp == 0) {
    const uint32_t holder = static_cast<uint32_t>(__cvta_generic_to_shared(&tmem_holder));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(holder), "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_holder;
  float scale = 1.0f;
  if (prev_norm) {
    double tot = 0.0;
    for (int i = 0; i < n_prev; ++i) tot += prev_norm[i];
    scale = tot > 0.0 ? float(1.0 / sqrt(tot)) : 1.0f;
  }
  double norm_acc = 0.0;

  const uint32_t ahi_s = static_cast<uint32_t>(__cvta_generic_to_shared(a_hi));
  const uint32_t alo_s = static_cast<uint32_t>(__cvta_generic_to_shared(a_lo));
  const uint32_t bhi_s = static_cast<uint32_t>(__cvta_generic_to_shared(b_hi));
  const uint32_t blo_s = static_cast<uint32_t>(__cvta_generic_to_shared(b_lo));

  uint32_t phase = 0;
  auto tile_base_of = [&](uint64_t tile) {
    const uint64_t mine = ((tile >> lane) & 1ull) ? lane_bit : 0ull;
    const uint32_t lo = __reduce_or_sync(0xffffffffu, uint32_t(mine));
    const uint32_t hi = __reduce_or_sync(0xffffffffu, uint32_t(mine >> 32));
    return uint64_t(lo) | (uint64_t(hi) << 32);
  };
  // tile base tb has no sub-cube bits, and sub-cube bit 0 is qubit 0, so the
  // pair (u, u + 1) is one 16-byte-aligned float4
  auto load_tile = [&](uint64_t tb, float4 (&v)[kLoadSteps]) {
    const float4* src4 = reinterpret_cast<const float4*>(reinterpret_cast<const float2*>(amp) + tb + t_addr);
#pragma unroll
    for (int i = 0; i < kLoadSteps; ++i) v[i] = __ldcs(src4 + (it_addr[(uint32_t(i) + g) & 15u] >> 1));
  };
  // the tiles two and three ahead are pulled into L2 meanwhile (no registers
  // or shared memory held), so the next loads meet L2 rather than DRAM latency
  auto prefetch_tile = [&](uint64_t tb) {
    const float4* src4 = reinterpret_cast<const float4*>(reinterpret_cast<const float2*>(amp) + tb + t_addr);
#pragma unroll
    for (int i = 0; i < kLoadSteps; ++i)
      asm volatile("prefetch.global.L2 [%0];\n" ::"l"(src4 + (it_addr[(uint32_t(i) + g) & 15u] >> 1)));
  };
  // HBM -> A_hi / A_lo (split), swizzled K-major rows; (re, im) = columns
  // (2j, 2j + 1) share one aligned 8-byte slot of a 16-byte chunk
  auto put = [&](uint32_t o0, float re, float im) {
    const float hr = tf32_rn(re), hi_ = tf32_rn(im);
    *reinterpret_cast<float2*>(a_hi + o0) = make_float2(hr, hi_);
    *reinterpret_cast<float2*>(a_lo + o0) = make_float2(tf32_rn(re - hr), tf32_rn(im - hi_));
  };
  // qubit 0 a column bit: the pair (u, u + 1) is columns (j, j + 1) of one
  // row, j even, i.e. one 16-byte chunk of the swizzled layout
  auto put2 = [&](uint32_t o0, float4 x) {
    const float4 h = make_float4(tf32_rn(x.x), tf32_rn(x.y), tf32_rn(x.z), tf32_rn(x.w));
    *reinterpret_cast<float4*>(a_hi + o0) = h;
    *reinterpret_cast<float4*>(a_lo + o0) =
        make_float4(tf32_rn(x.x - h.x), tf32_rn(x.y - h.y), tf32_rn(x.z - h.z), tf32_rn(x.w - h.w));
  };
  // Software pipeline over this CTA's tiles t0, t1, ... (two accumulators of
  // 64 TMEM columns).  While the epilogue warps drain tile t from one
  // accumulator, the loading warps split tile t+1 (loaded during the previous
  // round) into the operand planes, which the MMAs of tile t have released,
  // and issue its MMAs into the other accumulator; the HBM loads of tile t+2
  // follow, and the tiles after it are prefetched into L2.
  float4 v[kLoadSteps];
  // loading warps: operand split of the tile in v (writers make their shared
  // stores visible to the tensor core before the barrier)
  auto put_tile = [&]() {
    if (A.lane_over_j) {
#pragma unroll
      for (int i = 0; i < kLoadSteps; ++i) put2(op_t ^ it_op[(uint32_t(i) + g) & 15u], v[i]);
    } else {
#pragma unroll
      for (int i = 0; i < kLoadSteps; ++i) {
        const uint32_t o0 = op_t ^ it_op[(uint32_t(i) + g) & 15u];
        put(o0, v[i].x, v[i].y);
        put(o0 ^ op_h, v[i].z, v[i].w);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  };
  auto issue_mma = [&](uint32_t acc_col) {
    if (tid == 0) {
      uint32_t acc = 0;
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) {
        const uint32_t off = (kk >> 2) * kAtomBytes + (kk & 3) * 32;
        const uint32_t boff = (kk >> 2) * (64 * 128) + (kk & 3) * 32;
        mma_tf32(tmem + acc_col, umma_desc(ahi_s + off), umma_desc(bhi_s + boff), acc);
        acc = 1;
        mma_tf32(tmem + acc_col, umma_desc(ahi_s + off), umma_desc(blo_s + boff), 1);
        mma_tf32(tmem + acc_col, umma_desc(alo_s + off), umma_desc(bhi_s + boff), 1);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar_addr)
                   : "memory");
    }
  };
  // bounded wait for the last MMAs issued; false: the CTA gives up (error
  // flagged).  No MMA is issued after a wait that expired, and the MMAs it was
  // waiting for get one more bounded wait before the CTA leaves its tile loop
  // for the normal exit, which frees their TMEM accumulators.
  auto wait_mma = [&]() {
    uint32_t it = 0;
    bool done = false;
    while (!(done = mbar_try_wait(mbar_addr, phase)) && ++it < kWaitLimit) {
    }
    if (!done) {
      atomicExch(err, 1);
      abort_flag = 1;
      for (uint32_t j = 0; j < 4 * kWaitLimit && !mbar_try_wait(mbar_addr, phase); ++j) {
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    phase ^= 1u;
    return abort_flag == 0;
  };
  // epilogue warps: accumulator at column acc_col -> HBM; warp w reads lanes
  // 32 (w % 4) .. + 31 (row = tid % 128), all 64 fp32 columns in two halves
  auto epilogue = [&](uint64_t tb, uint32_t acc_col) {
    double tile_norm = 0.0;
    float2* out = reinterpret_cast<float2*>(amp) + tb + row_addr;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      uint32_t r[32];
      const uint32_t jb = uint32_t(half) * 16u;
      const uint32_t taddr = tmem + (uint32_t((warp & 3) * 32) << 16) + acc_col + 2u * jb;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
            "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      // when qubit 0 is fused, columns (j, j + 1) are adjacent amplitudes (16 bytes)
      if (A.lane_over_j) {
#pragma unroll
        for (int jj = 0; jj < 16; jj += 2) {
          const float4 o = make_float4(__uint_as_float(r[2 * jj]) * scale, __uint_as_float(r[2 * jj + 1]) * scale,
                                       __uint_as_float(r[2 * jj + 2]) * scale,
                                       __uint_as_float(r[2 * jj + 3]) * scale);
          tile_norm += double(o.x) * double(o.x) + double(o.y) * double(o.y) + double(o.z) * double(o.z) +
                       double(o.w) * double(o.w);
          __stcs(reinterpret_cast<float4*>(out + ctab[jb + uint32_t(jj)]), o);
        }
      } else {
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          const float2 o = make_float2(__uint_as_float(r[2 * jj]) * scale, __uint_as_float(r[2 * jj + 1]) * scale);
          tile_norm += double(o.x) * double(o.x) + double(o.y) * double(o.y);
          __stcs(out + ctab[jb + uint32_t(jj)], o);
        }
      }
    }
    norm_acc += tile_norm;
  };
  const uint64_t G = gridDim.x;
  uint64_t tile = blockIdx.x;
  if (tile < n_tiles) {
    if (loader) {
      load_tile(tile_base_of(tile), v);
      if (tile + G < n_tiles) prefetch_tile(tile_base_of(tile + G));
      if (tile + 2 * G < n_tiles) prefetch_tile(tile_base_of(tile + 2 * G));
      put_tile();
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    issue_mma(0);
    if (loader) {
      if (tile + G < n_tiles) load_tile(tile_base_of(tile + G), v);
      if (tile + 3 * G < n_tiles) prefetch_tile(tile_base_of(tile + 3 * G));
    }
    uint32_t cur = 0;  // TMEM column of the accumulator that holds `tile`
    bool ok = wait_mma();
    while (ok) {
      const uint64_t next = tile + G;
      if (loader) {
        if (next < n_tiles) {
          put_tile();  // tile `next`: the operand planes are free (the MMAs of `tile` are done)
          asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
          asm volatile("bar.sync 1, %0;\n" ::"n"(kProdThreads) : "memory");  // loading warps only
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          issue_mma(cur ^ 64u);
          if (next + G < n_tiles) load_tile(tile_base_of(next + G), v);
          if (next + 3 * G < n_tiles) prefetch_tile(tile_base_of(next + 3 * G));
        }
      } else {
        epilogue(tile_base_of(tile), cur);
      }
      if (next >= n_tiles) break;
      // orders this epilogue's TMEM reads before the next MMAs into `cur`, and
      // the MMAs of `next` before the next operand split
      ok = wait_mma();
      tile = next;
      cur ^= 64u;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  // per-CTA FP64 norm partial (fixed-order tree: warp shuffles, then warp 0)
  __shared__ double wsum[kFusedThreads / 32];
  double nsum = norm_acc;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nsum += __shfl_xor_sync(0xffffffffu, nsum, o);
  if (lane == 0) wsum[warp] = nsum;
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < kFusedThreads / 32; ++w) t += wsum[w];
    out_norm[blockIdx.x] = t;
  }
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(128));
}

// ---------------------------------------------------------------------------
// Plan management
// ---------------------------------------------------------------------------
struct FusedPlanImpl {
  int n = 0;
  std::vector<FusedGate> gates;
  std::vector<FusedArgs> args;
  float* d_bmats = nullptr;  // per gate: hi[64][64], lo[64][64]
  int norm_slots = 0;  // per-CTA norm partials per launch (the state holds two buffers, ping-pong)
};

static void real_embedding(const FusedGate& g, float* hi, float* lo) {
  for (int j = 0; j < 32; ++j)
    for (int k = 0; k < 32; ++k) {
      const cplx u = g.u[j * 32 + k];
      const double vals[2][2] = {{u.real(), -u.imag()}, {u.imag(), u.real()}};
      auto rn = [](float x) {
        uint32_t bits;
        std::memcpy(&bits, &x, 4);
        bits = (bits + 0x1000u) & 0xFFFFE000u;
        float h;
        std::memcpy(&h, &bits, 4);
        return h;
      };
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
          const float h = rn(float(vals[a][b]));
          const int row = 2 * j + a, col = 2 * k + b;
          hi[row * 64 + col] = h;
          lo[row * 64 + col] = rn(float(vals[a][b] - double(h)));
        }
    }
}

static FusedArgs make_args(const FusedGate& g, int n) {
  FusedArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = n;
  uint64_t F = 0;
  for (int i = 0; i < 5; ++i) { a.q[i] = g.q[i]; F |= 1ull << g.q[i]; }
  int ng = 0;
  uint64_t G = 0;
  for (int q = 0; q < n && ng < 7; ++q)
    if (!((F >> q) & 1)) { a.gq[ng++] = q; G |= 1ull << q; }
  a.ng = ng;
  // Row order of the group qubits.  The operand store of amplitude (row r,
  // column c) lands in the 8-byte bank slot (c & 1) | (((c >> 1) ^ r) & 7) << 1
  // of the 128-byte-swizzled layout, and the lanes of a warp run over qubits
  // 1..5.  Row bits 0..2 are given to lane qubits wherever the matching column
  // bit (c bits 1..3) is not a lane qubit, so that the lanes of one store phase
  // (a quarter warp for the 16-byte stores used when qubit 0 is a column bit,
  // a half warp for the 8-byte ones otherwise) hit distinct slots.
  {
    const int wmax = (F & 1ull) ? 3 : 4;  // lane qubits 1..wmax share one store phase
    auto in_w = [&](int q) { return q >= 1 && q <= wmax; };
    int order[7];
    bool used[7] = {false, false, false, false, false, false, false};
    int no = 0;
    for (int k = 0; k < 3 && k < ng; ++k) {
      const bool col_is_lane = k + 1 < 5 && in_w(a.q[k + 1]);
      int pick = -1;
      for (int i = 0; i < ng && pick < 0; ++i)
        if (!used[i] && in_w(a.gq[i]) != col_is_lane) pick = i;
      for (int i = 0; i < ng && pick < 0; ++i)
        if (!used[i]) pick = i;
      used[pick] = true;
      order[no++] = a.gq[pick];
    }
    for (int i = 0; i < ng; ++i)
      if (!used[i]) order[no++] = a.gq[i];
    for (int i = 0; i < ng; ++i) a.gq[i] = order[i];
  }
  int no = 0;
  for (int q = 0; q < n; ++q)
    if (!(((F | G) >> q) & 1)) a.qout[no++] = q;
  a.n_out = no;
  a.lane_over_j = (F & 1ull) ? 1 : 0;
  // Sub-cube bits: 0..5 are qubits 0..5 (16-byte pairs, lanes: 512 contiguous
  // bytes per warp), 6..7 the loading warps, 8..11 the load steps.  When column
  // bit 0 (the lowest fused qubit) is not a lane qubit it becomes step bit 0
  // and lane groups run the steps rotated, so that one store covers both
  // column parities.
  int nb = 0;
  for (int q = 0; q < n && nb < 12; ++q)
    if (((F | G) >> q) & 1) a.sub[nb++] = q;
  a.rot = 0;
  if (a.q[0] >= 6) {
    int at = -1;
    for (int b = 6; b < 12; ++b)
      if (a.sub[b] == a.q[0]) at = b;
    std::swap(a.sub[at], a.sub[8]);
    a.rot = 1;
  }
  for (int b = 0; b < 12; ++b) {
    const int q = a.sub[b];
    a.sub_row[b] = -1;
    a.sub_col[b] = -1;
    if ((F >> q) & 1) {
      for (int i = 0; i < 5; ++i)
        if (a.q[i] == q) a.sub_col[b] = i;
    } else {
      for (int i = 0; i < ng; ++i)
        if (a.gq[i] == q) a.sub_row[b] = i;
    }
  }
  return a;
}

bool fused_plan_stats(const std::vector<Op>& ops, int n, DType dt, PlanStats* stats) {
  if (dt != DType::C64 || n < 12) return false;
  std::vector<FusedGate> g = fuse_ops(ops, n);
  stats->passes = g.size();
  stats->ops = ops.size();
  stats->stages = g.size();
  stats->upload_bytes = g.size() * 2 * 64 * 64 * sizeof(float);
  return true;
}

bool fused_plan_build(const std::vector<Op>& ops, int n, DType dt, void** plan, PlanStats* stats) {
  *plan = nullptr;
  // complex64 only; 12 qubits minimum (5 fused + 7 group bits per 128-row tile)
  if (dt != DType::C64 || n < 12) return false;
  auto* p = new FusedPlanImpl();
  p->n = n;
  p->gates = fuse_ops(ops, n);
  const size_t G = p->gates.size();
  std::vector<float> host(std::max<size_t>(1, G) * 2 * 4096);
  for (size_t i = 0; i < G; ++i) {
    real_embedding(p->gates[i], host.data() + i * 8192, host.data() + i * 8192 + 4096);
    p->args.push_back(make_args(p->gates[i], n));
  }
  bool ok = cudaMalloc(reinterpret_cast<void**>(&p->d_bmats), host.size() * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMemcpy(p->d_bmats, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
  p->norm_slots = device_sms() * kFusedCtasPerSm;
  if (!ok) {
    fused_plan_free(p);
    return false;
  }
  stats->passes = G;
  stats->ops = ops.size();
  stats->stages = G;
  stats->upload_bytes = host.size() * sizeof(float);
  *plan = p;
  return true;
}

void fused_plan_free(void* plan) {
  auto* p = static_cast<FusedPlanImpl*>(plan);
  if (!p) return;
  if (p->d_bmats) cudaFree(p->d_bmats);
  delete p;
}

cudaError_t fused_run(void* plan, StateImpl* s, std::vector<cudaEvent_t>* events) {
  auto* p = static_cast<FusedPlanImpl*>(plan);
  if (!p || s->dt != DType::C64 || int(s->n) != p->n) return cudaErrorInvalidValue;
  // the shared-memory limit is a per-device attribute: set once per device
  static PerDeviceOnce<cudaError_t> attr;
  int dev = 0;
  cudaError_t ae = cudaGetDevice(&dev);
  if (ae != cudaSuccess) return ae;
  ae = attr.get(dev, [] { return cudaFuncSetAttribute(k_fused_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFused); },
                cudaErrorInvalidDevice);
  if (ae != cudaSuccess) return ae;
  // norm partials and expiry flag of this run: the state's scratch
  double* d_norm = nullptr;
  int* d_err = nullptr;
  if ((ae = state_run_scratch(s, 2 * size_t(p->norm_slots), &d_norm, &d_err)) != cudaSuccess) return ae;
  const int n = p->n;
  const uint64_t n_tiles = 1ull << (n - 12);
  const unsigned grid = unsigned(std::min<uint64_t>(n_tiles, uint64_t(p->norm_slots)));
  cudaError_t e = cudaSuccess;
  int prev_grid = 0;
  for (size_t i = 0; i < p->gates.size(); ++i) {
    double* outn = d_norm + (i & 1) * p->norm_slots;
    const double* prevn = i ? d_norm + ((i + 1) & 1) * p->norm_slots : nullptr;
    k_fused_apply<<<grid, kFusedThreads, kSmemFused, s->stream>>>(
        static_cast<float*>(s->amp), p->args[i], p->d_bmats + i * 8192, prevn, prev_grid, outn, n_tiles,
        d_err);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    prev_grid = int(grid);
    if (events) {
      cudaEvent_t ev;
      if ((e = cudaEventCreate(&ev)) != cudaSuccess) return e;
      events->push_back(ev);
      if ((e = cudaEventRecord(ev, s->stream)) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}


}  // namespace nqpu
