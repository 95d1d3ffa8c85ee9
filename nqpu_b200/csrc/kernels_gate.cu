// Per-gate kernels: one launch = one gate = one pass over the amplitudes the
// gate touches.  These are the B200 form of GateOperations' per-gate Rayon
// passes (R/lib.rs:617-1735) and of the C FFI's InternalQuantumState kernels
// (c_ffi.rs:268-535):
//   * work items enumerate exactly the index sets the reference enumerates with
//     insert_zero_bit(s) (R/lib.rs:575-630): zero bits inserted at the target
//     positions, one bits forced at the control positions, so a controlled gate
//     reads and writes only the amplitudes it changes (CNOT: S bytes, CZ: S/2);
//   * complex64 items are vectorised over qubit 0 with 128-bit float4 accesses
//     whenever qubit 0 is neither a target nor a control; complex128 amplitudes
//     are 128-bit double2 accesses;
//   * grid-stride loops with two items in flight per thread, grid sized to
//     the SM count.
#include "sv_device.cuh"
#include "kernels.h"

namespace nqpu {

template <typename Real>
__device__ __forceinline__ void load_m(const PGArgs& A, typename Tr<Real>::C* m, int cnt) {
  for (int i = 0; i < cnt; ++i) {
    m[i].x = Real(A.m[2 * i]);
    m[i].y = Real(A.m[2 * i + 1]);
  }
}

__device__ __forceinline__ uint64_t pg_expand(uint64_t w, const PGArgs& A) {
  uint64_t i = w;
#pragma unroll 1
  for (int j = 0; j < A.npos; ++j) i = insert_zero_bit(i, A.pos[j]);
  return i | A.setmask;
}

// ---- dense / X on one target ----------------------------------------------
// MODE 0: scalar amplitudes (complex128 always; complex64 when qubit 0 is a
//         control): item -> pair (i, i|2^t).
// MODE 1: complex64, target t >= 1, qubit 0 free: item -> float4 at i and at
//         i|2^t (two pairs).
// MODE 2: complex64, target 0: item -> one float4 holding the pair.
template <typename Real, int KIND, int MODE>
__global__ void __launch_bounds__(256) k_pg_1t(Real* __restrict__ amp, PGArgs A) {
  using C = typename Tr<Real>::C;
  C m[4];
  if (KIND == OP_U1) load_m<Real>(A, m, 4);
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t tbit = 1ull << A.t0;
  for (uint64_t w = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; w < A.n_items; w += 2 * stride) {
    const uint64_t w2 = w + stride;
    const bool has2 = w2 < A.n_items;
    const uint64_t i0 = pg_expand(w, A);
    const uint64_t i1 = has2 ? pg_expand(w2, A) : 0;
    if constexpr (MODE == 1) {
      float4* p = reinterpret_cast<float4*>(amp);
      float4 x0 = __ldcs(p + (i0 >> 1)), y0 = __ldcs(p + ((i0 | tbit) >> 1));
      float4 x1, y1;
      if (has2) { x1 = __ldcs(p + (i1 >> 1)); y1 = __ldcs(p + ((i1 | tbit) >> 1)); }
      auto op = [&](float4& x, float4& y) {
        float2 a0 = make_float2(x.x, x.y), a1 = make_float2(x.z, x.w);
        float2 b0 = make_float2(y.x, y.y), b1 = make_float2(y.z, y.w);
        if (KIND == OP_U1) {
          float2 na0 = cmac2(m[0], a0, m[1], b0), nb0 = cmac2(m[2], a0, m[3], b0);
          float2 na1 = cmac2(m[0], a1, m[1], b1), nb1 = cmac2(m[2], a1, m[3], b1);
          x = make_float4(na0.x, na0.y, na1.x, na1.y);
          y = make_float4(nb0.x, nb0.y, nb1.x, nb1.y);
        } else {
          float4 t = x; x = y; y = t;
        }
      };
      op(x0, y0);
      __stcs(p + (i0 >> 1), x0); __stcs(p + ((i0 | tbit) >> 1), y0);
      if (has2) { op(x1, y1); __stcs(p + (i1 >> 1), x1); __stcs(p + ((i1 | tbit) >> 1), y1); }
    } else if constexpr (MODE == 2) {
      float4* p = reinterpret_cast<float4*>(amp);
      float4 x0 = __ldcs(p + (i0 >> 1));
      float4 x1;
      if (has2) x1 = __ldcs(p + (i1 >> 1));
      auto op = [&](float4& x) {
        float2 a = make_float2(x.x, x.y), b = make_float2(x.z, x.w);
        if (KIND == OP_U1) {
          float2 na = cmac2(m[0], a, m[1], b), nb = cmac2(m[2], a, m[3], b);
          x = make_float4(na.x, na.y, nb.x, nb.y);
        } else {
          x = make_float4(x.z, x.w, x.x, x.y);
        }
      };
      op(x0);
      __stcs(p + (i0 >> 1), x0);
      if (has2) { op(x1); __stcs(p + (i1 >> 1), x1); }
    } else {
      C* p = reinterpret_cast<C*>(amp);
      C a0 = p[i0], b0 = p[i0 | tbit];
      C a1, b1;
      if (has2) { a1 = p[i1]; b1 = p[i1 | tbit]; }
      auto op = [&](C& a, C& b) {
        if (KIND == OP_U1) {
          C na = cmac2(m[0], a, m[1], b), nb = cmac2(m[2], a, m[3], b);
          a = na; b = nb;
        } else {
          C t = a; a = b; b = t;
        }
      };
      op(a0, b0);
      p[i0] = a0; p[i0 | tbit] = b0;
      if (has2) { op(a1, b1); p[i1] = a1; p[i1 | tbit] = b1; }
    }
  }
}

// ---- dense / swap on two targets ------------------------------------------
// VEC: complex64 with qubit 0 free: four float4 per item (two quads).
template <typename Real, int KIND, bool VEC>
__global__ void __launch_bounds__(256) k_pg_2t(Real* __restrict__ amp, PGArgs A) {
  using C = typename Tr<Real>::C;
  C m[16];
  if (KIND == OP_U2) load_m<Real>(A, m, 16);
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t b0 = 1ull << A.t0, b1 = 1ull << A.t1;
  for (uint64_t w = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; w < A.n_items; w += stride) {
    const uint64_t i = pg_expand(w, A);
    if constexpr (VEC) {
      float4* p = reinterpret_cast<float4*>(amp);
      float4 v0 = __ldcs(p + (i >> 1)), v1 = __ldcs(p + ((i | b0) >> 1));
      float4 v2 = __ldcs(p + ((i | b1) >> 1)), v3 = __ldcs(p + ((i | b0 | b1) >> 1));
      if (KIND == OP_U2) {
        float2 xa[4] = {make_float2(v0.x, v0.y), make_float2(v1.x, v1.y), make_float2(v2.x, v2.y),
                        make_float2(v3.x, v3.y)};
        float2 xb[4] = {make_float2(v0.z, v0.w), make_float2(v1.z, v1.w), make_float2(v2.z, v2.w),
                        make_float2(v3.z, v3.w)};
        float2 ya[4], yb[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          ya[r] = cmac4(m + 4 * r, xa[0], xa[1], xa[2], xa[3]);
          yb[r] = cmac4(m + 4 * r, xb[0], xb[1], xb[2], xb[3]);
        }
        v0 = make_float4(ya[0].x, ya[0].y, yb[0].x, yb[0].y);
        v1 = make_float4(ya[1].x, ya[1].y, yb[1].x, yb[1].y);
        v2 = make_float4(ya[2].x, ya[2].y, yb[2].x, yb[2].y);
        v3 = make_float4(ya[3].x, ya[3].y, yb[3].x, yb[3].y);
      } else {
        float4 t = v1; v1 = v2; v2 = t;
      }
      __stcs(p + (i >> 1), v0); __stcs(p + ((i | b0) >> 1), v1);
      __stcs(p + ((i | b1) >> 1), v2); __stcs(p + ((i | b0 | b1) >> 1), v3);
    } else {
      C* p = reinterpret_cast<C*>(amp);
      C x0 = p[i], x1 = p[i | b0], x2 = p[i | b1], x3 = p[i | b0 | b1];
      if (KIND == OP_U2) {
        p[i] = cmac4(m + 0, x0, x1, x2, x3);
        p[i | b0] = cmac4(m + 4, x0, x1, x2, x3);
        p[i | b1] = cmac4(m + 8, x0, x1, x2, x3);
        p[i | b0 | b1] = cmac4(m + 12, x0, x1, x2, x3);
      } else {
        p[i | b0] = x2;
        p[i | b1] = x1;
      }
    }
  }
}

// ---- elementwise phases (D1, D2 over all amplitudes; PH on a masked subset)
// PH: items enumerate only amplitudes with all mask bits set.
template <typename Real, int KIND, bool VEC>
__global__ void __launch_bounds__(256) k_pg_elem(Real* __restrict__ amp, PGArgs A) {
  using C = typename Tr<Real>::C;
  C m[4];
  load_m<Real>(A, m, KIND == OP_D2 ? 4 : (KIND == OP_D1 ? 2 : 1));
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t cm = A.cmask;
  auto phase = [&](uint64_t idx, C v) -> C {
    if (KIND == OP_PH) return cmul(m[0], v);
    if ((idx & cm) != cm) return v;
    int s = int((idx >> A.t0) & 1);
    if (KIND == OP_D2) s |= int((idx >> A.t1) & 1) << 1;
    return cmul(m[s], v);
  };
  for (uint64_t w = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; w < A.n_items; w += 2 * stride) {
    const uint64_t w2 = w + stride;
    const bool has2 = w2 < A.n_items;
    const uint64_t i0 = pg_expand(w, A);
    const uint64_t i1 = has2 ? pg_expand(w2, A) : 0;
    if constexpr (VEC) {
      float4* p = reinterpret_cast<float4*>(amp);
      float4 x0 = __ldcs(p + (i0 >> 1));
      float4 x1;
      if (has2) x1 = __ldcs(p + (i1 >> 1));
      auto op = [&](uint64_t i, float4& x) {
        float2 a = phase(i, make_float2(x.x, x.y));
        float2 b = phase(i | 1, make_float2(x.z, x.w));
        x = make_float4(a.x, a.y, b.x, b.y);
      };
      op(i0, x0);
      __stcs(p + (i0 >> 1), x0);
      if (has2) { op(i1, x1); __stcs(p + (i1 >> 1), x1); }
    } else {
      C* p = reinterpret_cast<C*>(amp);
      C a0 = p[i0];
      C a1;
      if (has2) a1 = p[i1];
      p[i0] = phase(i0, a0);
      if (has2) p[i1] = phase(i1, a1);
    }
  }
}

static unsigned pg_grid(uint64_t items, int num_sms) {
  const uint64_t max_blocks = uint64_t(num_sms) * 8;
  uint64_t need = (items + 255) / 256;
  if (need < 1) need = 1;
  return unsigned(need < max_blocks ? need : max_blocks);
}

// Host-side lowering of one op to a per-gate launch.
template <typename Real>
static cudaError_t launch_pg_t(Real* amp, int n, const Op& op, cudaStream_t s, int num_sms) {
  PGArgs A{};
  for (int i = 0; i < 16; ++i) {
    A.m[2 * i] = op.m[i].real();
    A.m[2 * i + 1] = op.m[i].imag();
  }
  A.t0 = op.t0;
  A.t1 = op.t1;
  const bool c64 = sizeof(Real) == 4;
  uint64_t ctrl = op.ctrl_mask();
  std::vector<int> pos;
  auto finish = [&](bool insert_bit0) {
    if (insert_bit0) pos.push_back(0);
    std::sort(pos.begin(), pos.end());
    pos.erase(std::unique(pos.begin(), pos.end()), pos.end());
    A.npos = int(pos.size());
    for (int i = 0; i < A.npos; ++i) A.pos[i] = pos[i];
    A.n_items = (1ull << n) >> A.npos;
  };
  const unsigned blk = 256;
  switch (op.kind) {
    case OP_U1:
    case OP_X1: {
      pos.push_back(op.t0);
      for (int i = 0; i < op.nctrl; ++i) pos.push_back(op.ctrl[i]);
      A.setmask = ctrl;
      if constexpr (sizeof(Real) == 4) {
        if (op.t0 == 0 && !(ctrl & 1)) {
          finish(false);
          unsigned g = pg_grid(A.n_items, num_sms);
          if (op.kind == OP_U1) k_pg_1t<Real, OP_U1, 2><<<g, blk, 0, s>>>(amp, A);
          else k_pg_1t<Real, OP_X1, 2><<<g, blk, 0, s>>>(amp, A);
          break;
        }
        if (!(ctrl & 1) && n >= 2) {
          finish(true);
          unsigned g = pg_grid(A.n_items, num_sms);
          if (op.kind == OP_U1) k_pg_1t<Real, OP_U1, 1><<<g, blk, 0, s>>>(amp, A);
          else k_pg_1t<Real, OP_X1, 1><<<g, blk, 0, s>>>(amp, A);
          break;
        }
      }
      {
        finish(false);
        unsigned g = pg_grid(A.n_items, num_sms);
        if (op.kind == OP_U1) k_pg_1t<Real, OP_U1, 0><<<g, blk, 0, s>>>(amp, A);
        else k_pg_1t<Real, OP_X1, 0><<<g, blk, 0, s>>>(amp, A);
      }
      break;
    }
    case OP_U2:
    case OP_SW: {
      pos.push_back(op.t0);
      pos.push_back(op.t1);
      for (int i = 0; i < op.nctrl; ++i) pos.push_back(op.ctrl[i]);
      A.setmask = ctrl;
      const bool vec = c64 && op.t0 != 0 && op.t1 != 0 && !(ctrl & 1);
      finish(vec);
      unsigned g = pg_grid(A.n_items, num_sms);
      if constexpr (sizeof(Real) == 4) {
        if (vec) {
          if (op.kind == OP_U2) k_pg_2t<Real, OP_U2, true><<<g, blk, 0, s>>>(amp, A);
          else k_pg_2t<Real, OP_SW, true><<<g, blk, 0, s>>>(amp, A);
          break;
        }
      }
      if (op.kind == OP_U2) k_pg_2t<Real, OP_U2, false><<<g, blk, 0, s>>>(amp, A);
      else k_pg_2t<Real, OP_SW, false><<<g, blk, 0, s>>>(amp, A);
      break;
    }
    case OP_PH: {
      // only amplitudes with t0 and every control set change
      pos.push_back(op.t0);
      for (int i = 0; i < op.nctrl; ++i) pos.push_back(op.ctrl[i]);
      A.setmask = ctrl | (1ull << op.t0);
      const bool vec = c64 && !(A.setmask & 1) && n >= 1;
      finish(vec);
      unsigned g = pg_grid(A.n_items, num_sms);
      if constexpr (sizeof(Real) == 4) {
        if (vec) { k_pg_elem<Real, OP_PH, true><<<g, blk, 0, s>>>(amp, A); break; }
      }
      k_pg_elem<Real, OP_PH, false><<<g, blk, 0, s>>>(amp, A);
      break;
    }
    case OP_D1:
    case OP_D2: {
      // controls restrict the touched set; diagonal qubits stay free
      for (int i = 0; i < op.nctrl; ++i) pos.push_back(op.ctrl[i]);
      A.setmask = ctrl;
      A.cmask = 0;
      const bool vec = c64 && !(ctrl & 1) && n >= 1;
      finish(vec);
      unsigned g = pg_grid(A.n_items, num_sms);
      if constexpr (sizeof(Real) == 4) {
        if (vec) {
          if (op.kind == OP_D1) k_pg_elem<Real, OP_D1, true><<<g, blk, 0, s>>>(amp, A);
          else k_pg_elem<Real, OP_D2, true><<<g, blk, 0, s>>>(amp, A);
          break;
        }
      }
      if (op.kind == OP_D1) k_pg_elem<Real, OP_D1, false><<<g, blk, 0, s>>>(amp, A);
      else k_pg_elem<Real, OP_D2, false><<<g, blk, 0, s>>>(amp, A);
      break;
    }
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_pergate(DType dt, void* amp, int n, const Op& op, cudaStream_t s, int num_sms) {
  if (dt == DType::C64) return launch_pg_t<float>(static_cast<float*>(amp), n, op, s, num_sms);
  return launch_pg_t<double>(static_cast<double*>(amp), n, op, s, num_sms);
}

}  // namespace nqpu
