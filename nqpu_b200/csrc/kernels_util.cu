// Elementwise state kernels: basis-state init (QuantumState::new / reset,
// R/lib.rs:331 and c_ffi.rs:233), scaling/renormalisation, measurement
// collapse (c_ffi.rs:537-566, GateOperations::reset_qubit R/lib.rs:1705),
// probabilities (R/lib.rs:354) and dtype conversion.
#include "sv_device.cuh"
#include "kernels.h"

namespace nqpu {

static unsigned ew_grid(uint64_t items, int num_sms) {
  const uint64_t max_blocks = uint64_t(num_sms) * 8;
  uint64_t need = (items + 255) / 256;
  if (need < 1) need = 1;
  return unsigned(need < max_blocks ? need : max_blocks);
}

template <typename Real>
__global__ void k_set_basis(Real* __restrict__ amp, uint64_t dim2, uint64_t index) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < dim2; i += stride)
    amp[i] = (i == 2 * index) ? Real(1) : Real(0);
}

template <typename Real>
__global__ void k_scale(Real* __restrict__ amp, uint64_t dim2, Real f) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < dim2; i += stride)
    amp[i] *= f;
}

template <typename Real>
__global__ void k_collapse(Real* __restrict__ amp, uint64_t dim, int q, int keep, Real f) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < dim; i += stride) {
    const bool k = int((i >> q) & 1) == keep;
    amp[2 * i] = k ? amp[2 * i] * f : Real(0);
    amp[2 * i + 1] = k ? amp[2 * i + 1] * f : Real(0);
  }
}

template <typename Real>
__global__ void k_probs(const Real* __restrict__ amp, uint64_t dim, double* __restrict__ out) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < dim; i += stride) {
    const double r = amp[2 * i], m = amp[2 * i + 1];
    out[i] = r * r + m * m;
  }
}

template <typename RS, typename RD>
__global__ void k_convert(const RS* __restrict__ src, RD* __restrict__ dst, uint64_t dim2) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < dim2; i += stride)
    dst[i] = RD(src[i]);
}

cudaError_t launch_set_basis(DType dt, void* amp, int n, uint64_t index, cudaStream_t s, int num_sms) {
  const uint64_t dim2 = 2ull << n;
  if (dt == DType::C64) k_set_basis<float><<<ew_grid(dim2, num_sms), 256, 0, s>>>(static_cast<float*>(amp), dim2, index);
  else k_set_basis<double><<<ew_grid(dim2, num_sms), 256, 0, s>>>(static_cast<double*>(amp), dim2, index);
  return cudaGetLastError();
}

cudaError_t launch_scale(DType dt, void* amp, int n, double factor, cudaStream_t s, int num_sms) {
  const uint64_t dim2 = 2ull << n;
  if (dt == DType::C64) k_scale<float><<<ew_grid(dim2, num_sms), 256, 0, s>>>(static_cast<float*>(amp), dim2, float(factor));
  else k_scale<double><<<ew_grid(dim2, num_sms), 256, 0, s>>>(static_cast<double*>(amp), dim2, factor);
  return cudaGetLastError();
}

cudaError_t launch_collapse(DType dt, void* amp, int n, int q, int keep, double factor,
                            cudaStream_t s, int num_sms) {
  const uint64_t dim = 1ull << n;
  if (dt == DType::C64) k_collapse<float><<<ew_grid(dim, num_sms), 256, 0, s>>>(static_cast<float*>(amp), dim, q, keep, float(factor));
  else k_collapse<double><<<ew_grid(dim, num_sms), 256, 0, s>>>(static_cast<double*>(amp), dim, q, keep, factor);
  return cudaGetLastError();
}

cudaError_t launch_probabilities(DType dt, const void* amp, uint64_t count, double* out, cudaStream_t s, int num_sms) {
  const uint64_t dim = count;
  if (dt == DType::C64) k_probs<float><<<ew_grid(dim, num_sms), 256, 0, s>>>(static_cast<const float*>(amp), dim, out);
  else k_probs<double><<<ew_grid(dim, num_sms), 256, 0, s>>>(static_cast<const double*>(amp), dim, out);
  return cudaGetLastError();
}

cudaError_t launch_convert(DType sdt, const void* src, DType ddt, void* dst, uint64_t count, cudaStream_t s, int num_sms) {
  const uint64_t dim2 = 2ull * count;
  const unsigned g = ew_grid(dim2, num_sms);
  if (sdt == DType::C64 && ddt == DType::C128) k_convert<float, double><<<g, 256, 0, s>>>(static_cast<const float*>(src), static_cast<double*>(dst), dim2);
  else if (sdt == DType::C128 && ddt == DType::C64) k_convert<double, float><<<g, 256, 0, s>>>(static_cast<const double*>(src), static_cast<float*>(dst), dim2);
  else if (sdt == DType::C64) k_convert<float, float><<<g, 256, 0, s>>>(static_cast<const float*>(src), static_cast<float*>(dst), dim2);
  else k_convert<double, double><<<g, 256, 0, s>>>(static_cast<const double*>(src), static_cast<double*>(dst), dim2);
  return cudaGetLastError();
}

}  // namespace nqpu
