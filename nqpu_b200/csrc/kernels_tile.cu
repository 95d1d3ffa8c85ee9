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
#include "device_once.h"
#include "kernels.h"
#include "tile_device.cuh"

namespace nqpu {

// Dynamic shared memory: [tile buffer 0 | tile buffer 1 | hi_off table
// (2^(k-c) <= kHiOffEntries u64) | stage tables (kMaxPassStages x kStageTabWords u32)].
// MINB = 1: one persistent CTA per SM; while the stages of tile i run on one
// buffer, the cp.async copies of tile i+1 stream into the other.  MINB > 1:
// MINB CTAs per SM with one buffer each hide each other's copies.  Each thread
// holds 16 vectors, so a CTA has 2^KMAX / (16 x amplitudes per vector) threads.
template <typename Real, int KMAX, int MINB>
__global__ void __launch_bounds__(1 << (KMAX - Tr<Real>::kVecBit - 4), MINB)
    k_tile_pass(Real* __restrict__ amp, const PassRec* __restrict__ passes,
                const StageRec* __restrict__ stages, const TileOp<Real>* __restrict__ ops,
                int pass_idx, uint64_t n_tiles) {
  using T = Tr<Real>;
  using V = typename T::V;
  constexpr int VB = T::kVecBit;
  constexpr uint32_t kMaxVec = 1u << (KMAX - VB);
  constexpr int kThreads = int(kMaxVec) / kVecPerThread;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr bool kDoubleBuffer = (MINB == 1);
  V* buf0 = reinterpret_cast<V*>(smem_raw);
  V* buf1 = kDoubleBuffer ? buf0 + kMaxVec : buf0;
  uint64_t* hi_off = reinterpret_cast<uint64_t*>(smem_raw + (kDoubleBuffer ? 2 : 1) * sizeof(V) * kMaxVec);
  uint32_t* tabs = reinterpret_cast<uint32_t*>(hi_off + kHiOffEntries);
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
  build_pass_tabs<Real>(P, stages, tabs);  // ends with a barrier
  const uint32_t lowmask = (1u << c) - 1u;

  // HBM -> shared, asynchronous (consecutive threads take consecutive vectors).
  auto issue_load = [&](uint64_t tile, V* dst) {
    const uint64_t base = tile_base(P, tile);
#pragma unroll
    for (int i = 0; i < kVecPerThread; ++i) {
      const uint32_t u = tid + i * kThreads;
      if (u < nvec) {
        const uint32_t t = u << VB;
        const uint64_t g = base + (t & lowmask) + hi_off[t >> c];
        cp_async16(dst + swz(u), amp + 2 * g);
      }
    }
  };

  uint64_t tile = blockIdx.x;
  if (kDoubleBuffer) {
    if (tile < n_tiles) issue_load(tile, buf0);
    cp_async_commit();
  }
  for (int it = 0; tile < n_tiles; ++it, tile += gridDim.x) {
    V* sv = (it & 1) ? buf1 : buf0;
    const uint64_t next = tile + gridDim.x;
    if (kDoubleBuffer) {
      if (next < n_tiles) issue_load(next, (it & 1) ? buf0 : buf1);
    } else {
      issue_load(tile, sv);  // single buffer: the other CTA on the SM hides the latency
    }
    cp_async_commit();
    if (kDoubleBuffer) cp_async_wait1();  // everything but the newest group (the prefetch) has landed
    else cp_async_wait0();
    __syncthreads();

    const uint64_t base = tile_base(P, tile);
    uint32_t ext = 0;
    for (int j = 0; j < P.n_ext; ++j)
      if ((base >> P.ext[j]) & 1ull) ext |= 1u << (k + j);

    run_tile_stages<Real>(sv, P, tabs, ops, ext);

    // shared -> HBM
#pragma unroll
    for (int i = 0; i < kVecPerThread; ++i) {
      const uint32_t u = tid + i * kThreads;
      if (u < nvec) {
        const uint32_t t = u << VB;
        const uint64_t g = base + (t & lowmask) + hi_off[t >> c];
        __stcs(reinterpret_cast<V*>(amp + 2 * g), sv[swz(u)]);
      }
    }
    __syncthreads();  // this buffer is refilled by the prefetch issued next iteration
  }
}

// Largest tile (bits) per dtype: 64 KB of amplitudes.
template <typename Real>
constexpr int tile_kmax_full() { return sizeof(Real) == 4 ? 13 : 12; }

template <typename Real, int KMAX>
static size_t tile_smem_bytes(int minb) {
  using V = typename Tr<Real>::V;
  return (minb == 1 ? 2 : 1) * sizeof(V) * (size_t(1) << (KMAX - Tr<Real>::kVecBit)) +
         sizeof(uint64_t) * kHiOffEntries + sizeof(uint32_t) * kMaxPassStages * kStageTabWords;
}

// CTA configuration of the tiled pass kernel per dtype (CTAs per SM):
//   1: one 64 KB-tile CTA per SM, double-buffered (cp.async prefetch of the next tile);
//   2: two 64 KB-tile CTAs per SM, one buffer each;
//   4: four CTAs per SM on 32 KB tiles (one tile bit fewer, half the threads):
//      more independent CTAs to overlap each other's barriers and copies, at
//      the price of more passes.
// Plans are built for the configuration's tile size (tile_kmax_for).
// Defaults measured on B200 (28-qubit brickwork): complex64 runs fastest with
// four 32 KB-tile CTAs per SM, complex128 with one double-buffered CTA (its
// 2-CTA build spills registers).
static int g_tile_minb[2] = {4, 1};

void tile_config_set(DType dt, int minb) {
  g_tile_minb[dt == DType::C64 ? 0 : 1] = (minb == 4) ? 4 : (minb == 2) ? 2 : 1;
}
int tile_config_get(DType dt) { return g_tile_minb[dt == DType::C64 ? 0 : 1]; }

template <typename Real, int KMAX, int MINB>
cudaError_t launch_tile_pass_cfg(Real* amp, const PassRec& host_pass, const PassRec* d_passes,
                                 const StageRec* d_stages, const TileOp<Real>* d_ops, int pass_idx,
                                 cudaStream_t stream, int num_sms) {
  // a plan built for larger tiles than this kernel holds must not run on it,
  // nor one whose tables exceed the shared-memory copies
  if (host_pass.k > KMAX || host_pass.k < 1 || host_pass.k - host_pass.c > kHiOffBits ||
      host_pass.stage_end - host_pass.stage_begin > kMaxPassStages)
    return cudaErrorInvalidValue;
  auto kern = k_tile_pass<Real, KMAX, MINB>;
  constexpr int kThreads = (1 << (KMAX - Tr<Real>::kVecBit)) / kVecPerThread;
  // shared memory of this launch: the tile buffer(s), the high-offset table and
  // the stage tables of this pass only (more CTAs fit when passes are short)
  const size_t smem_max = tile_smem_bytes<Real, KMAX>(MINB);
  const size_t smem = smem_max - sizeof(uint32_t) * kStageTabWords *
                                     size_t(kMaxPassStages - (host_pass.stage_end - host_pass.stage_begin));
  // the shared-memory limit is a per-device attribute: set once per device
  static PerDeviceOnce<cudaError_t> attr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = attr.get(dev, [&] { return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_max)); },
               cudaErrorInvalidDevice);
  if (e != cudaSuccess) return e;
  const uint64_t n_tiles = 1ull << host_pass.n_out;
  const uint64_t max_ctas = uint64_t(num_sms) * MINB;
  const unsigned grid = unsigned(n_tiles < max_ctas ? n_tiles : max_ctas);
  kern<<<grid, kThreads, smem, stream>>>(amp, d_passes, d_stages, d_ops, pass_idx, n_tiles);
  return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_tile_pass_t(Real* amp, int n, const PassRec& host_pass, const PassRec* d_passes,
                               const StageRec* d_stages, const TileOp<Real>* d_ops, int pass_idx,
                               cudaStream_t stream, int num_sms) {
  (void)n;
  constexpr int K = tile_kmax_full<Real>();
  switch (g_tile_minb[sizeof(Real) == 4 ? 0 : 1]) {
    case 4:
      return launch_tile_pass_cfg<Real, K - 1, 4>(amp, host_pass, d_passes, d_stages, d_ops, pass_idx, stream,
                                                  num_sms);
    case 2:
      return launch_tile_pass_cfg<Real, K, 2>(amp, host_pass, d_passes, d_stages, d_ops, pass_idx, stream, num_sms);
    default:
      return launch_tile_pass_cfg<Real, K, 1>(amp, host_pass, d_passes, d_stages, d_ops, pass_idx, stream, num_sms);
  }
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

int tile_kmax_for(DType dt) {
  const int full = dt == DType::C64 ? 13 : 12;
  return tile_config_get(dt) == 4 ? full - 1 : full;
}

}  // namespace nqpu
