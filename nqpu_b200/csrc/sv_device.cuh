// Device-side helpers shared by the statevector kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "sv_types.h"

namespace nqpu {

// Complex scalar and 128-bit vector types per precision.
//   complex64 : amplitude float2,  vector float4  = 2 amplitudes (index bit 0 pair)
//   complex128: amplitude double2, vector double2 = 1 amplitude
template <typename Real> struct Tr;
template <> struct Tr<float> {
  using C = float2;
  using V = float4;
  static constexpr int kAmpsPerVec = 2;
  static constexpr int kVecBit = 1;  // log2(amps per vector)
};
template <> struct Tr<double> {
  using C = double2;
  using V = double2;
  static constexpr int kAmpsPerVec = 1;
  static constexpr int kVecBit = 0;
};

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// a*x + b*y for complex a, b, x, y (the 2x2 row product).
template <typename C>
__device__ __forceinline__ C cmac2(C a, C x, C b, C y) {
  C r;
  r.x = a.x * x.x - a.y * x.y + b.x * y.x - b.y * y.y;
  r.y = a.x * x.y + a.y * x.x + b.x * y.y + b.y * y.x;
  return r;
}
template <typename C>
__device__ __forceinline__ C cmac4(const C* m, C x0, C x1, C x2, C x3) {
  C r;
  r.x = m[0].x * x0.x - m[0].y * x0.y + m[1].x * x1.x - m[1].y * x1.y +
        m[2].x * x2.x - m[2].y * x2.y + m[3].x * x3.x - m[3].y * x3.y;
  r.y = m[0].x * x0.y + m[0].y * x0.x + m[1].x * x1.y + m[1].y * x1.x +
        m[2].x * x2.y + m[2].y * x2.x + m[3].x * x3.y + m[3].y * x3.x;
  return r;
}

// Packed complex64 arithmetic (sm_100 FFMA2: one instruction on a float2
// register pair).  A complex coefficient m is held as p = (re, re) and
// q = (-im, im), so m * x = p * x + q * (x.im, x.re): two packed operations per
// complex product instead of four scalar ones.  The swapped operand is always
// the second multiplicand.
struct PackedC {
  float2 p, q;
};
__device__ __forceinline__ PackedC pack_coef(float2 m) {
  return PackedC{make_float2(m.x, m.x), make_float2(-m.y, m.y)};
}
__device__ __forceinline__ float2 swap_ri(float2 v) { return make_float2(v.y, v.x); }
// m * x
__device__ __forceinline__ float2 pcmul(const PackedC& m, float2 x) {
  return __ffma2_rn(m.q, swap_ri(x), __fmul2_rn(m.p, x));
}
// m0 * x + m1 * y (the 2x2 row product)
__device__ __forceinline__ float2 pcmac2(const PackedC& m0, float2 x, const PackedC& m1, float2 y) {
  float2 t = __fmul2_rn(m0.p, x);
  t = __ffma2_rn(m0.q, swap_ri(x), t);
  t = __ffma2_rn(m1.p, y, t);
  return __ffma2_rn(m1.q, swap_ri(y), t);
}

__device__ __forceinline__ uint64_t insert_zero_bit(uint64_t v, int bit) {
  uint64_t lo = v & ((1ull << bit) - 1);
  return lo | ((v >> bit) << (bit + 1));
}

template <typename V> __device__ __forceinline__ V ldg_v(const V* p) { return __ldg(p); }
template <typename V> __device__ __forceinline__ V ldcs_v(const V* p) { return __ldcs(p); }

}  // namespace nqpu
