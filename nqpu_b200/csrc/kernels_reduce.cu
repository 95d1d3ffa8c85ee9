// FP64 reductions over the statevector: all <Z_q> in one pass, inner products
// (fidelity), Pauli-string expectations and shot sampling.
//
// Reference semantics: QuantumState::expectation_z / fidelity /
// expectation_pauli_string / sample (R/lib.rs:388-560) and the C FFI's
// expectation_z / sample (c_ffi.rs:576-620).  The reference runs each of these
// as a serial loop per qubit or per term; here every reduction is one coalesced
// pass with FP64 accumulation: per-thread Kahan sums, warp-shuffle trees, and a
// final single-block FP64 combine, so results are deterministic for a given
// state and launch shape.
#include "sv_device.cuh"
#include "kernels.h"

namespace nqpu {

struct KSum {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {
    double y = x - c;
    double t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kRedThreads = 256;
constexpr int kRedVecPerThread = 16;  // a segment = 256 * 16 vectors

template <typename Real>
__device__ __forceinline__ void vec_probs(const typename Tr<Real>::V& v, double* p);
template <>
__device__ __forceinline__ void vec_probs<float>(const float4& v, double* p) {
  p[0] = double(v.x) * double(v.x) + double(v.y) * double(v.y);
  p[1] = double(v.z) * double(v.z) + double(v.w) * double(v.w);
}
template <>
__device__ __forceinline__ void vec_probs<double>(const double2& v, double* p) {
  p[0] = v.x * v.x + v.y * v.y;
}

// Layout of the zsums scratch (doubles, kernels.h):
//   [0, nblk*kBlkVals)            per-block low-bit partials
//   [kZsMaxBlocks*kBlkVals, + nseg) per-segment totals
constexpr int kBlkVals = kZsBlkVals;  // tot, bit0(c64), 8 thread bits, 4 j bits, (pad)
static_assert(kZsSegVecs == uint64_t(kRedThreads) * kRedVecPerThread, "segment size");

template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
    k_zsums(const Real* __restrict__ amp, int n, uint64_t nseg, double* __restrict__ blk_part,
            double* __restrict__ seg_part) {
  using V = typename Tr<Real>::V;
  constexpr int VB = Tr<Real>::kVecBit;
  constexpr int APV = Tr<Real>::kAmpsPerVec;
  const uint64_t nvec_total = (1ull << n) >> VB;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  KSum tot, b0;
  KSum jb[4];
  const V* vp = reinterpret_cast<const V*>(amp);
  static_assert(kRedThreads == 256, "segment total sums 8 warps");
  __shared__ double seg_red[kRedThreads / 32];
  for (uint64_t seg = blockIdx.x; seg < nseg; seg += gridDim.x) {
    const uint64_t vbase = seg * (kRedThreads * kRedVecPerThread);
    V v[kRedVecPerThread];
#pragma unroll
    for (int j = 0; j < kRedVecPerThread; ++j) {
      const uint64_t vi = vbase + tid + j * kRedThreads;
      if (vi < nvec_total) v[j] = __ldcs(vp + vi);
    }
    double segp = 0.0;
#pragma unroll
    for (int j = 0; j < kRedVecPerThread; ++j) {
      const uint64_t vi = vbase + tid + j * kRedThreads;
      if (vi < nvec_total) {
        double p[2];
        vec_probs<Real>(v[j], p);
        double pv = p[0];
        if (APV == 2) {
          pv += p[1];
          b0.add(p[1]);
        }
        tot.add(pv);
        segp += pv;
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (j & (1 << q)) jb[q].add(pv);
      }
    }
    segp = warp_sum(segp);
    if (lane == 0) seg_red[warp] = segp;
    __syncthreads();
    if (tid == 0)
      seg_part[seg] = ((seg_red[0] + seg_red[1]) + (seg_red[2] + seg_red[3])) +
                      ((seg_red[4] + seg_red[5]) + (seg_red[6] + seg_red[7]));
    __syncthreads();
  }
  // Per-block partials of the low bits: thread bits come from the per-thread totals.
  __shared__ double red[kRedThreads / 32][kBlkVals];
  double vals[kBlkVals];
  const double t = tot.s;
  vals[0] = t;
  vals[1] = b0.s;
#pragma unroll
  for (int b = 0; b < 8; ++b) vals[2 + b] = ((tid >> b) & 1) ? t : 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) vals[10 + q] = jb[q].s;
  vals[14] = vals[15] = 0.0;
#pragma unroll
  for (int i = 0; i < kBlkVals; ++i) vals[i] = warp_sum(vals[i]);
  if (lane == 0)
    for (int i = 0; i < kBlkVals; ++i) red[warp][i] = vals[i];
  __syncthreads();
  if (tid < kBlkVals) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) s += red[w][tid];
    blk_part[blockIdx.x * kBlkVals + tid] = s;
  }
}

// Final combine: one block.  Low bits from block partials, high bits from
// segment partials (segment index bit b <-> amplitude bit H + b).
template <int VB>
__global__ void __launch_bounds__(1024)
    k_zsums_final(int n, int nblk, uint64_t nseg, int H, const double* __restrict__ blk_part,
                  double* __restrict__ seg_part, double* __restrict__ out) {
  __shared__ double sh[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto block_sum = [&](double v) -> double {
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
      r = (lane < int(blockDim.x / 32)) ? sh[lane] : 0.0;
      r = warp_sum(r);
    }
    return r;  // valid in thread 0
  };
  // low-bit values: index 0 = total, then per amplitude bit
  // complex64: amp bit 0 -> vals[1]; amp bits 1..8 -> vals[2..9]; bits 9..12 -> vals[10..13]
  // complex128: amp bits 0..7 -> vals[2..9]; bits 8..11 -> vals[10..13]
  for (int vi = 0; vi < 14; ++vi) {
    double s = 0.0;
    for (int b = tid; b < nblk; b += blockDim.x) s += blk_part[b * kBlkVals + vi];
    s = block_sum(s);
    if (tid == 0) {
      int qbit;
      if (vi == 0) qbit = -1;
      else if (vi == 1) qbit = (VB == 1) ? 0 : -2;
      else if (vi < 10) qbit = VB + (vi - 2);
      else qbit = VB + 8 + (vi - 10);
      if (qbit == -1) out[0] = s;
      else if (qbit >= 0 && qbit < n && qbit < H) out[1 + qbit] = s;
    }
  }
  // High bits: nseg is a power of two (2^(n-H)).  Fold the segment totals in
  // half, top bit first: at level b the upper half A[2^b .. 2^(b+1)) sums to the
  // weight of amplitude bit H + b, and A[i] += A[i + 2^b] leaves A[0 .. 2^b)
  // indexed by the lower segment bits.  In place: at each level every i is
  // read and written by one thread only; block_sum's barriers order the levels.
  double* A = seg_part;
  for (int b = n - H - 1; b >= 0; --b) {
    const uint64_t half = 1ull << b;
    KSum acc;
    for (uint64_t i = tid; i < half; i += blockDim.x) {
      const double u = A[i + half];
      acc.add(u);
      A[i] += u;
    }
    const double s = block_sum(acc.s);
    if (tid == 0) out[1 + H + b] = s;
  }
}

static uint64_t seg_vecs() { return kZsSegVecs; }

size_t reduce_scratch_bytes(int n) {
  // worst case complex128: one vector per amplitude
  size_t zs = sizeof(double) * zsums_scratch_doubles(n);
  size_t samp = sizeof(double) * (2 * ((1ull << n) / 4096 + 2) + 64);
  size_t inner = sizeof(double) * (2 * 4096 + 64);
  return std::max(zs, std::max(samp, inner)) + 4096;
}

template <typename Real>
static cudaError_t zsums_t(const Real* amp, int n, double* scratch, double* out, cudaStream_t s,
                           int num_sms) {
  constexpr int VB = Tr<Real>::kVecBit;
  const uint64_t nvec = (1ull << n) >> VB;
  const uint64_t nvec_eff = nvec ? nvec : 1;
  const uint64_t nseg = (nvec_eff + seg_vecs() - 1) / seg_vecs();
  int nblk = int(std::min<uint64_t>(nseg, uint64_t(num_sms) * 4));
  nblk = std::min(nblk, kZsMaxBlocks);
  double* blk_part = scratch;
  double* seg_part = scratch + size_t(kZsMaxBlocks) * kBlkVals;
  // segment = 4096 vectors = 2^(12 + VB) amplitudes
  const int H = 12 + VB;
  k_zsums<Real><<<nblk, kRedThreads, 0, s>>>(amp, n, nseg, blk_part, seg_part);
  k_zsums_final<VB><<<1, 1024, 0, s>>>(n, nblk, nseg, H, blk_part, seg_part, out);
  return cudaGetLastError();
}

cudaError_t launch_zsums(DType dt, const void* amp, int n, double* scratch, double* out,
                         cudaStream_t s, int num_sms) {
  if (dt == DType::C64) return zsums_t<float>(static_cast<const float*>(amp), n, scratch, out, s, num_sms);
  return zsums_t<double>(static_cast<const double*>(amp), n, scratch, out, s, num_sms);
}

// ---- inner product ----------------------------------------------------------
template <typename RA, typename RB>
__global__ void __launch_bounds__(kRedThreads)
    k_inner(const RA* __restrict__ a, const RB* __restrict__ b, uint64_t dim,
            double* __restrict__ part) {
  KSum re, im;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < dim; i += stride) {
    const double ar = a[2 * i], ai = a[2 * i + 1];
    const double br = b[2 * i], bi = b[2 * i + 1];
    re.add(ar * br + ai * bi);
    im.add(ar * bi - ai * br);
  }
  __shared__ double sh[2][kRedThreads / 32];
  double r = warp_sum(re.s), m = warp_sum(im.s);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { sh[0][warp] = r; sh[1][warp] = m; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sr = 0, sm = 0;
    for (int w = 0; w < kRedThreads / 32; ++w) { sr += sh[0][w]; sm += sh[1][w]; }
    part[2 * blockIdx.x] = sr;
    part[2 * blockIdx.x + 1] = sm;
  }
}

__global__ void k_sum_pairs(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  // single warp, deterministic order
  double r = 0, m = 0;
  for (int i = threadIdx.x; i < nblk; i += 32) { r += part[2 * i]; m += part[2 * i + 1]; }
  r = warp_sum(r);
  m = warp_sum(m);
  if (threadIdx.x == 0) { out[0] = r; out[1] = m; }
}

cudaError_t launch_inner(DType dta, const void* a, DType dtb, const void* b, int n, double* scratch,
                         double* out, cudaStream_t s, int num_sms) {
  const uint64_t dim = 1ull << n;
  int nblk = int(std::min<uint64_t>((dim + kRedThreads - 1) / kRedThreads, uint64_t(num_sms) * 8));
  nblk = std::max(1, std::min(nblk, 4096));
  if (dta == DType::C64 && dtb == DType::C64)
    k_inner<float, float><<<nblk, kRedThreads, 0, s>>>(static_cast<const float*>(a), static_cast<const float*>(b), dim, scratch);
  else if (dta == DType::C64)
    k_inner<float, double><<<nblk, kRedThreads, 0, s>>>(static_cast<const float*>(a), static_cast<const double*>(b), dim, scratch);
  else if (dtb == DType::C64)
    k_inner<double, float><<<nblk, kRedThreads, 0, s>>>(static_cast<const double*>(a), static_cast<const float*>(b), dim, scratch);
  else
    k_inner<double, double><<<nblk, kRedThreads, 0, s>>>(static_cast<const double*>(a), static_cast<const double*>(b), dim, scratch);
  k_sum_pairs<<<1, 32, 0, s>>>(scratch, nblk, out);
  return cudaGetLastError();
}

// ---- Pauli string expectation (R/lib.rs:465) --------------------------------
// coeff(i) = i^ny * (-1)^popcount(i & zmask); j = i ^ xmask;
// result = sum_i Re(conj(a_i) * coeff(i) * a_j).
template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
    k_pauli(const Real* __restrict__ amp, uint64_t dim, uint64_t xmask, uint64_t zmask, int ny,
            double* __restrict__ part) {
  KSum acc;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < dim; i += stride) {
    const uint64_t j = i ^ xmask;
    const double ar = amp[2 * i], ai = amp[2 * i + 1];
    const double br = amp[2 * j], bi = amp[2 * j + 1];
    // c = i^ny * sign
    double cr, ci;
    switch (ny & 3) {
      case 0: cr = 1; ci = 0; break;
      case 1: cr = 0; ci = 1; break;
      case 2: cr = -1; ci = 0; break;
      default: cr = 0; ci = -1; break;
    }
    if (__popcll(i & zmask) & 1) { cr = -cr; ci = -ci; }
    const double pr = cr * br - ci * bi;
    const double pi = cr * bi + ci * br;
    acc.add(ar * pr + ai * pi);
  }
  __shared__ double sh[kRedThreads / 32];
  double r = warp_sum(acc.s);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sr = 0;
    for (int w = 0; w < kRedThreads / 32; ++w) sr += sh[w];
    part[2 * blockIdx.x] = sr;
    part[2 * blockIdx.x + 1] = 0.0;
  }
}

cudaError_t launch_pauli(DType dt, const void* amp, int n, uint64_t xmask, uint64_t zmask,
                         uint64_t ymask, double* scratch, double* out, cudaStream_t s,
                         int num_sms) {
  const uint64_t dim = 1ull << n;
  int nblk = int(std::min<uint64_t>((dim + kRedThreads - 1) / kRedThreads, uint64_t(num_sms) * 8));
  nblk = std::max(1, std::min(nblk, 4096));
  const int ny = __builtin_popcountll(ymask);
  if (dt == DType::C64)
    k_pauli<float><<<nblk, kRedThreads, 0, s>>>(static_cast<const float*>(amp), dim, xmask, zmask, ny, scratch);
  else
    k_pauli<double><<<nblk, kRedThreads, 0, s>>>(static_cast<const double*>(amp), dim, xmask, zmask, ny, scratch);
  k_sum_pairs<<<1, 32, 0, s>>>(scratch, nblk, out);
  return cudaGetLastError();
}

// ---- sampling ---------------------------------------------------------------
constexpr int kSampSegBits = 12;  // 4096 amplitudes per CDF segment

template <typename Real>
__global__ void __launch_bounds__(256)
    k_seg_probs(const Real* __restrict__ amp, uint64_t dim, uint64_t nseg, int segbits,
                double* __restrict__ seg_sum) {
  __shared__ double sh[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t seglen = 1ull << segbits;
  for (uint64_t sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
    double acc = 0.0;
    for (uint64_t k = threadIdx.x; k < seglen; k += blockDim.x) {
      const uint64_t i = sg * seglen + k;
      if (i < dim) {
        const double ar = amp[2 * i], ai = amp[2 * i + 1];
        acc += ar * ar + ai * ai;
      }
    }
    acc = warp_sum(acc);
    if (lane == 0) sh[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0;
      for (int w = 0; w < 8; ++w) t += sh[w];
      seg_sum[sg] = t;
    }
    __syncthreads();
  }
}

// Inclusive scan of seg_sum into seg_incl (single block, FP64, deterministic).
__global__ void __launch_bounds__(1024)
    k_seg_scan(const double* __restrict__ seg_sum, uint64_t nseg, double* __restrict__ seg_incl) {
  __shared__ double sh[1024];
  const uint64_t per = (nseg + blockDim.x - 1) / blockDim.x;
  const uint64_t b = threadIdx.x * per;
  const uint64_t e = b + per < nseg ? b + per : nseg;
  double local = 0.0;
  for (uint64_t i = b; i < e; ++i) local += seg_sum[i];
  sh[threadIdx.x] = local;
  __syncthreads();
  // Hillis-Steele inclusive scan over the 1024 chunk totals
  for (int off = 1; off < 1024; off <<= 1) {
    double v = (threadIdx.x >= unsigned(off)) ? sh[threadIdx.x - off] : 0.0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  double run = threadIdx.x ? sh[threadIdx.x - 1] : 0.0;
  for (uint64_t i = b; i < e; ++i) {
    run += seg_sum[i];
    seg_incl[i] = run;
  }
}

// One warp per shot.
template <typename Real>
__global__ void __launch_bounds__(256)
    k_sample(const Real* __restrict__ amp, uint64_t dim, int segbits, uint64_t nseg,
             const double* __restrict__ seg_sum, const double* __restrict__ seg_incl,
             const double* __restrict__ u, uint32_t shots, uint64_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint64_t warp_id = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t sh = warp_id; sh < shots; sh += nwarps) {
    const double r = u[sh];
    // first segment whose inclusive prefix exceeds r
    uint64_t lo = 0, hi = nseg;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (seg_incl[mid] > r) hi = mid; else lo = mid + 1;
    }
    uint64_t result = dim - 1;
    if (lo < nseg) {
      double run = seg_incl[lo] - seg_sum[lo];
      bool found = false;
      for (uint64_t sg = lo; sg < nseg && !found; ++sg) {
        if (sg != lo) run = seg_incl[sg] - seg_sum[sg];
        const uint64_t s0 = sg << segbits;
        const uint64_t s1 = (s0 + (1ull << segbits)) < dim ? s0 + (1ull << segbits) : dim;
        for (uint64_t base = s0; base < s1; base += 32) {
          const uint64_t i = base + lane;
          double p = 0.0;
          if (i < s1) {
            const double ar = amp[2 * i], ai = amp[2 * i + 1];
            p = ar * ar + ai * ai;
          }
          // inclusive warp scan
          double sc = p;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            double t = __shfl_up_sync(0xffffffffu, sc, o);
            if (lane >= o) sc += t;
          }
          const double cum = run + sc;
          const unsigned hit = __ballot_sync(0xffffffffu, (i < s1) && (r < cum));
          if (hit) {
            result = base + (__ffs(hit) - 1);
            found = true;
            break;
          }
          run += __shfl_sync(0xffffffffu, sc, 31);
        }
      }
    }
    if (lane == 0) out[sh] = result;
  }
}

cudaError_t launch_sample(DType dt, const void* amp, int n, const double* d_uniforms,
                          uint32_t shots, double* scratch, uint64_t* d_out, cudaStream_t s,
                          int num_sms) {
  const uint64_t dim = 1ull << n;
  const int segbits = n < kSampSegBits ? n : kSampSegBits;
  const uint64_t nseg = dim >> segbits;
  double* seg_sum = scratch;
  double* seg_incl = scratch + nseg + 1;
  const int g1 = int(std::min<uint64_t>(nseg, uint64_t(num_sms) * 8));
  if (dt == DType::C64)
    k_seg_probs<float><<<g1, 256, 0, s>>>(static_cast<const float*>(amp), dim, nseg, segbits, seg_sum);
  else
    k_seg_probs<double><<<g1, 256, 0, s>>>(static_cast<const double*>(amp), dim, nseg, segbits, seg_sum);
  k_seg_scan<<<1, 1024, 0, s>>>(seg_sum, nseg, seg_incl);
  if (shots == 0) return cudaGetLastError();
  const uint64_t warps = shots;
  const int g2 = int(std::max<uint64_t>(1, std::min<uint64_t>((warps * 32 + 255) / 256, uint64_t(num_sms) * 8)));
  if (dt == DType::C64)
    k_sample<float><<<g2, 256, 0, s>>>(static_cast<const float*>(amp), dim, segbits, nseg, seg_sum, seg_incl, d_uniforms, shots, d_out);
  else
    k_sample<double><<<g2, 256, 0, s>>>(static_cast<const double*>(amp), dim, segbits, nseg, seg_sum, seg_incl, d_uniforms, shots, d_out);
  return cudaGetLastError();
}

}  // namespace nqpu
