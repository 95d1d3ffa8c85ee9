// All-<Z_i> reduction for callers that cannot allocate device memory.
//
// Some callers of this library run where cudaMalloc is not available to them:
// code executing while a CUDA stream is being captured into a graph (allocation
// calls are illegal during capture), plugins hosted inside another runtime that
// owns the device memory pool, or real-time loops that must not block on the
// driver's allocator.  nqpu_expectation_z_all_noalloc serves them: the caller
// passes its own device amplitude buffer, its own device output buffer and its
// stream, and the reduction's scratch space comes from a fixed array in device
// global memory that is part of this library's module (loaded once per GPU and
// kept until the process exits).
//
// The scratch array is a __device__ symbol.  Host code cannot use its name as a
// device address (in host code the name is a host-side shadow), so the first
// call on each device, with that device current, resolves the real address
// with cudaGetSymbolAddress and caches it.  That first call should therefore
// happen before the caller starts capturing a stream.  All calls share the one
// array: two calls whose kernels overlap on the GPU race on it.  Nothing in the
// array has to start at zero: every partial sum the reduction reads is written
// earlier in the same call.
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/nqpu_b200.h"
#include "engine.h"
#include "kernels.h"

namespace nqpu {

// Scratch bound: per-block partials (1024 x 16) + per-segment partials for
// 2^27 128-bit vectors (32768 segments, room for 8 doubles each as the
// reduction's scratch layout reserves) + the n+1 sums.
constexpr int kNoAllocMaxVecLog2 = 27;
constexpr size_t kNoAllocScratchDoubles = 1024 * 16 + (size_t(1) << (kNoAllocMaxVecLog2 - 12)) * 8 + 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Resolve the device address of the scratch array for the current device.
cudaError_t scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}
}  // namespace

// <Z_q> = sum |a|^2 - 2 * sum_{bit q set} |a|^2
__global__ void k_z_from_sums(const double* __restrict__ sums, int n, double* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) out[q] = sums[0] - 2.0 * sums[1 + q];
}

}  // namespace nqpu

using namespace nqpu;

extern "C" NqpuError nqpu_expectation_z_all_noalloc(const void* d_amplitudes, uint32_t num_qubits,
                                                    NqpuDtype dtype, double* d_out, void* cuda_stream) {
  if (!d_amplitudes || !d_out) return NQPU_NULL_POINTER;
  if (dtype != NQPU_C64 && dtype != NQPU_C128) return NQPU_INVALID_PARAMETER;
  if (reinterpret_cast<uintptr_t>(d_amplitudes) % 16 != 0) return NQPU_INVALID_PARAMETER;  // 128-bit loads
  if (num_qubits == 0 || num_qubits > uint32_t(kMaxQubits)) return NQPU_INVALID_PARAMETER;
  const DType dt = dtype == NQPU_C64 ? DType::C64 : DType::C128;
  // 128-bit vectors in the state: complex64 packs two amplitudes per vector
  const int vec_log2 = int(num_qubits) - (dt == DType::C64 ? 1 : 0);
  if (vec_log2 > kNoAllocMaxVecLog2) return NQPU_INVALID_PARAMETER;  // beyond the fixed scratch
  if (!device_ready()) return NQPU_SIMULATION_FAILED;
  double* scratch = nullptr;
  if (scratch_for_current_device(&scratch) != cudaSuccess) return NQPU_SIMULATION_FAILED;
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  double* sums = scratch + (kNoAllocScratchDoubles - 64);  // n+1 <= 35 doubles at the end
  cudaError_t e = launch_zsums(dt, d_amplitudes, int(num_qubits), scratch, sums, st, device_sms());
  if (e != cudaSuccess) return NQPU_SIMULATION_FAILED;
  k_z_from_sums<<<1, 64, 0, st>>>(sums, int(num_qubits), d_out);
  if (cudaGetLastError() != cudaSuccess) return NQPU_SIMULATION_FAILED;
  return NQPU_OK;
}
