// Batched executor: many circuits of different sizes in one persistent launch.
//
// A device work queue (an array of tasks plus an atomic cursor) is consumed by
// a persistent grid of CTAs.  Task kinds:
//   * small circuit (n <= small_max): the whole state lives in one CTA's shared
//     memory (2^13 complex64 = 64 KB at most).  It is initialised to |0..0> in
//     shared memory, every register stage of the circuit's single tiled pass
//     runs there, and <H> is evaluated from shared memory: no HBM traffic for
//     the state at all.
//   * pass tile (c, p, t): tile t of pass p of a larger circuit whose state is
//     in the HBM arena.  Pass 0 synthesises |0..0> instead of loading.  Before
//     starting, the CTA waits until all tiles of pass p-1 of circuit c are done
//     (per-pass completion counters); after storing, it increments pass p's
//     counter.
//   * measure tile (c, t): after the last pass, tile t (amplitudes
//     [t*2^m, (t+1)*2^m), m = min(13, n)) contributes to <H> = sum_i J_i <Z_i Z_{i+1}> +
//     sum_i h_i <X_i>; per-tile FP64 partials are summed in tile order by the
//     CTA that finishes the circuit's last measure tile (deterministic result).
// The host orders the queue so that every task depends only on tasks queued
// before it, and the grid is no larger than the number of co-resident CTAs, so
// the waits always end; they are bounded anyway and set an error flag.
//
// Per-amplitude gate arithmetic is the tiled pass kernel's (run_tile_stages).
// Observable: the Ising energy of the batching configuration; the diagonal part
// uses byte lookup tables of bond sums, sum_i J_i z_i z_{i+1} = Jtot - 2 sum of
// J_i over the set bits of x ^ (x >> 1).
#include "batch.h"
#include "device_once.h"
#include "kernels.h"
#include "tile_device.cuh"

namespace nqpu {

constexpr int kBatchK = 13;                       // complex64 tile bits
constexpr uint32_t kBatchVec = 1u << (kBatchK - 1);

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// CTA-wide wait until *ctr >= target, at most `limit` polls; returns false on
// timeout (and flags the error for every CTA).
__device__ __forceinline__ bool wait_counter(const uint32_t* ctr, uint32_t target, uint32_t limit, int* err,
                                             int* s_flag) {
  if (threadIdx.x == 0) {
    uint32_t it = 0;
    bool ok = true;
    while (ld_acquire(ctr) < target) {
      // give up on an expired limit, or at once when another CTA already failed
      if (++it >= limit || ld_acquire(reinterpret_cast<const uint32_t*>(err)) != 0) {
        ok = false;
        atomicExch(err, 2);
        break;
      }
      __nanosleep(64);
    }
    *s_flag = ok ? 1 : 0;
  }
  __syncthreads();
  return *s_flag != 0;
}

__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < int(blockDim.x / 32); ++w) t += red[w];
  return t;  // valid in thread 0
}

// Ising-energy contribution of the amplitudes of a shared-memory tile whose
// local index covers the qubits 0..k-1 contiguously; `gbase` is the global
// index of local amplitude 0.  In-tile X partners come from shared memory;
// partners of qubits >= k are read from HBM (`state`, coherent L2 loads).
__device__ __forceinline__ double ising_tile(const float4* __restrict__ sv, int k, int n, uint64_t gbase,
                                             const float2* __restrict__ state, const double* lut,
                                             const double* hq, double jtot) {
  const uint32_t nvec = 1u << (k - 1);
  const uint64_t smask = (n >= 2) ? ((1ull << (n - 1)) - 1) : 0;
  double acc = 0.0;
  for (uint32_t u = threadIdx.x; u < nvec; u += blockDim.x) {
    const float4 v = sv[swz(u)];
    const float2 a[2] = {make_float2(v.x, v.y), make_float2(v.z, v.w)};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t xl = (u << 1) | h;
      const uint64_t x = gbase | xl;
      const double ar = a[h].x, ai = a[h].y;
      const double p = ar * ar + ai * ai;
      const uint64_t s = (x ^ (x >> 1)) & smask;
      const double d = jtot - 2.0 * (lut[s & 255] + lut[256 + ((s >> 8) & 255)] + lut[512 + ((s >> 16) & 255)]);
      acc += p * d;
      for (int i = 0; i < k; ++i) {
        if ((xl >> i) & 1u) continue;
        const uint32_t yl = xl | (1u << i);
        const float4 w = sv[swz(yl >> 1)];
        const float br = (yl & 1u) ? w.z : w.x, bi = (yl & 1u) ? w.w : w.y;
        acc += 2.0 * hq[i] * (ar * double(br) + ai * double(bi));
      }
      for (int i = k; i < n; ++i) {
        if ((x >> i) & 1ull) continue;
        const float2 b = __ldcg(state + (x | (1ull << i)));
        acc += 2.0 * hq[i] * (ar * double(b.x) + ai * double(b.y));
      }
    }
  }
  return acc;
}

__global__ void __launch_bounds__(kTileThreads, 2)
    k_batch(float* __restrict__ arena, const BatchCirc* __restrict__ circs, const BatchTask* __restrict__ tasks,
            uint32_t n_tasks, const PassRec* __restrict__ passes, const StageRec* __restrict__ stages,
            const TileOp<float>* __restrict__ ops, const double* __restrict__ obs, uint32_t* __restrict__ counters,
            double* __restrict__ partials, double* __restrict__ results, uint32_t* __restrict__ cursor,
            int* __restrict__ err, uint32_t spin_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* sv = reinterpret_cast<float4*>(smem_raw);
  uint64_t* hi_off = reinterpret_cast<uint64_t*>(smem_raw + sizeof(float4) * kBatchVec);
  double* lut = reinterpret_cast<double*>(hi_off + kHiOffEntries);  // 3 x 256 bond-sum tables
  double* hq = lut + 768;                                           // h_i, i < n
  uint32_t* tabs = reinterpret_cast<uint32_t*>(hq + 64);            // stage tables of the current pass
  __shared__ PassRec P;
  __shared__ int s_pass;  // global index of the pass whose tables are loaded (-1: none)
  __shared__ uint32_t s_task;
  __shared__ int s_flag;
  __shared__ double red[kTileThreads / 32];
  const int tid = threadIdx.x;

  auto load_obs = [&](const BatchCirc& C, double* jtot_out) {
    const double* J = obs + C.obs_base;
    const double* h = J + (C.n - 1);
    for (int i = tid; i < 768; i += blockDim.x) {
      const int tbl = i >> 8, byte = i & 255;
      double s = 0.0;
      for (int b = 0; b < 8; ++b) {
        const int bond = tbl * 8 + b;
        if (((byte >> b) & 1) && bond < C.n - 1) s += J[bond];
      }
      lut[i] = s;
    }
    for (int i = tid; i < C.n; i += blockDim.x) hq[i] = h[i];
    double jt = 0.0;
    for (int i = 0; i < C.n - 1; ++i) jt += J[i];
    *jtot_out = jt;
  };
  auto init_tile = [&](uint32_t nvec, bool one) {
    for (uint32_t u = tid; u < nvec; u += blockDim.x)
      sv[swz(u)] = (one && u == 0) ? make_float4(1.f, 0.f, 0.f, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
  };
  // Pass record, high-offset table and stage tables; consecutive tasks of the
  // same pass on this CTA reuse them.
  auto load_pass = [&](const BatchCirc& C, int p) {
    const int gp = C.pass_base + p;
    if (s_pass == gp) return;  // uniform: every thread read s_pass after the last barrier
    const int32_t* src = reinterpret_cast<const int32_t*>(passes + gp);
    int32_t* dst = reinterpret_cast<int32_t*>(&P);
    for (int i = tid; i < int(sizeof(PassRec) / 4); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    const int nhi = P.k - P.c;
    for (int hh = tid; hh < (1 << nhi); hh += blockDim.x) {
      uint64_t off = 0;
      for (int j = 0; j < nhi; ++j)
        if ((hh >> j) & 1) off |= 1ull << P.qhi[j];
      hi_off[hh] = off;
    }
    build_pass_tabs<float>(P, stages, tabs);  // ends with a barrier
    if (tid == 0) s_pass = gp;
    __syncthreads();
  };
  if (tid == 0) s_pass = -1;
  __syncthreads();

  for (;;) {
    if (tid == 0) {
      // stop handing out work once any CTA reported an error
      s_task = ld_acquire(reinterpret_cast<const uint32_t*>(err)) != 0 ? n_tasks : atomicAdd(cursor, 1u);
    }
    __syncthreads();
    const uint32_t ti = s_task;
    __syncthreads();  // s_task is rewritten by the next fetch
    if (ti >= n_tasks) break;
    const BatchTask T = tasks[ti];
    const BatchCirc C = circs[T.circ];

    if (T.phase < 0) {
      // ---- whole small circuit in shared memory ----
      load_pass(C, 0);
      const uint32_t nvec = 1u << (P.k - 1);
      init_tile(nvec, true);
      __syncthreads();
      run_tile_stages<float, true>(sv, P, tabs, ops, 0u);
      double jtot;
      load_obs(C, &jtot);
      __syncthreads();
      const double part = ising_tile(sv, C.n, C.n, 0, nullptr, lut, hq, jtot);
      const double e = block_sum(part, red);
      if (tid == 0) results[C.result] = e;
      __syncthreads();
      continue;
    }

    float2* state = reinterpret_cast<float2*>(arena) + C.amp_off;
    if (T.phase < C.n_passes) {
      // ---- one tile of one pass ----
      load_pass(C, T.phase);
      if (T.phase > 0) {
        const uint32_t need = 1u << passes[C.pass_base + T.phase - 1].n_out;
        if (!wait_counter(counters + C.done_base + T.phase - 1, need, spin_limit, err, &s_flag)) continue;
      }
      const int k = P.k, c = P.c;
      const uint32_t nvec = 1u << (k - 1);
      const uint32_t lowmask = (1u << c) - 1u;
      const uint64_t base = tile_base(P, T.tile);
      uint32_t ext = 0;
      for (int j = 0; j < P.n_ext; ++j)
        if ((base >> P.ext[j]) & 1ull) ext |= 1u << (k + j);
      if (T.phase == 0) {
        init_tile(nvec, base == 0);
      } else {
        for (uint32_t u = tid; u < nvec; u += blockDim.x) {
          const uint32_t t = u << 1;
          const uint64_t g = base + (t & lowmask) + hi_off[t >> c];
          cp_async16(sv + swz(u), state + g);
        }
        cp_async_commit();
        cp_async_wait0();
      }
      __syncthreads();
      run_tile_stages<float, true>(sv, P, tabs, ops, ext);
      for (uint32_t u = tid; u < nvec; u += blockDim.x) {
        const uint32_t t = u << 1;
        const uint64_t g = base + (t & lowmask) + hi_off[t >> c];
        __stcg(reinterpret_cast<float4*>(state + g), sv[swz(u)]);
      }
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        atomicAdd(counters + C.done_base + T.phase, 1u);
      }
      continue;
    }

    // ---- one measurement tile ----
    {
      const uint32_t need = 1u << passes[C.pass_base + C.n_passes - 1].n_out;
      if (!wait_counter(counters + C.done_base + C.n_passes - 1, need, spin_limit, err, &s_flag)) continue;
    }
    double jtot;
    load_obs(C, &jtot);
    const uint64_t gbase = uint64_t(T.tile) << C.meas_k;
    const uint32_t mvec = 1u << (C.meas_k - 1);
    for (uint32_t u = tid; u < mvec; u += blockDim.x) cp_async16(sv + swz(u), state + gbase + 2 * u);
    cp_async_commit();
    cp_async_wait0();
    __syncthreads();
    const double part = ising_tile(sv, C.meas_k, C.n, gbase, state, lut, hq, jtot);
    const double e = block_sum(part, red);
    if (tid == 0) {
      partials[C.part_base + T.tile] = e;
      __threadfence();
      const uint32_t prev = atomicAdd(counters + C.done_base + C.n_passes, 1u);
      if (prev + 1 == uint32_t(C.meas_tiles)) {
        __threadfence();
        double tot = 0.0;
        for (int i = 0; i < C.meas_tiles; ++i) tot += __ldcg(partials + C.part_base + i);
        results[C.result] = tot;
      }
    }
    __syncthreads();
  }
}

size_t batch_smem_bytes() {
  return sizeof(float4) * kBatchVec + sizeof(uint64_t) * kHiOffEntries + sizeof(double) * (768 + 64) +
         sizeof(uint32_t) * kMaxPassStages * kStageTabWords;
}

cudaError_t launch_batch(const BatchLaunch& L, cudaStream_t s) {
  const size_t smem = batch_smem_bytes();
  // the shared-memory limit is a per-device attribute: set once per device
  static PerDeviceOnce<cudaError_t> attr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = attr.get(dev, [&] { return cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)); },
               cudaErrorInvalidDevice);
  if (e != cudaSuccess) return e;
  k_batch<<<L.grid, kTileThreads, smem, s>>>(L.arena, L.circs, L.tasks, L.n_tasks, L.passes, L.stages, L.ops,
                                            L.obs, L.counters, L.partials, L.results, L.cursor, L.err,
                                            L.spin_limit ? L.spin_limit : kBatchSpinLimit);
  return cudaGetLastError();
}

}  // namespace nqpu
