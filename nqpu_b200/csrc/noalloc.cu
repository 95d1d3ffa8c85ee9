// All-<Z_i> reduction for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc themselves or through
// us: plugins hosted inside another runtime that owns the device memory pool
// (its allocator must be the only one, or memory it has reserved would be
// taken from under it), and real-time loops that must not block on the
// driver's allocator.  nqpu_expectation_z_all_noalloc serves them:
// the caller passes its own device amplitude buffer, its own device output
// buffer and its stream, and the reduction's scratch space comes from a fixed
// array in device global memory that is part of this library's module (loaded
// once per GPU and kept until the process exits).
//
// The scratch array is a __device__ symbol.  Host code cannot use its name as a
// device address (in host code the name is a host-side shadow), so the first
// call on each device, with that device current, resolves the real address
// with cudaGetSymbolAddress and caches it with the device's SM count.  That
// first call should therefore happen before the caller starts capturing a
// stream.  The address belongs to the device's primary context (the one the
// runtime API uses); it is not valid in other driver-API contexts, nor after
// cudaDeviceReset.  All calls share the one array: two calls whose kernels
// overlap on the GPU race on it.  Nothing in the array has to start at zero:
// every partial sum the reduction reads is written earlier in the same call.
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/nqpu_b200.h"
#include "device_once.h"
#include "engine.h"
#include "kernels.h"

namespace nqpu {

// Largest state: 2^27 128-bit vectors (complex64 up to 28 qubits, complex128
// up to 27).  The array holds the reduction's scratch for that size (its layout
// comes from zsums_scratch_doubles) plus 64 doubles at the end for the n+1 sums.
constexpr int kNoAllocMaxVecLog2 = 27;
constexpr size_t kNoAllocSumSlots = 64;
constexpr size_t kNoAllocScratchDoubles = zsums_scratch_doubles(kNoAllocMaxVecLog2) + kNoAllocSumSlots;
static_assert(kNoAllocSumSlots >= size_t(kMaxQubits) + 1, "room for the n+1 sums");
static_assert(kNoAllocScratchDoubles * sizeof(double) <= (size_t(3) << 20), "modest fixed footprint");

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

namespace {
struct DeviceScratch {
  double* addr = nullptr;
  int sms = 0;
  cudaError_t err = cudaSuccess;
};

// Device address of the scratch array and SM count of the current device,
// resolved once per device.
cudaError_t scratch_for_current_device(DeviceScratch* out) {
  static PerDeviceOnce<DeviceScratch> once;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  DeviceScratch bad;
  bad.err = cudaErrorInvalidDevice;
  *out = once.get(dev, [dev] {
    DeviceScratch d;
    void* p = nullptr;
    d.err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (d.err == cudaSuccess) d.err = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    if (d.err == cudaSuccess && d.sms <= 0) d.err = cudaErrorInvalidDevice;
    d.addr = static_cast<double*>(p);
    return d;
  }, bad);
  return out->err;
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
  DeviceScratch ds;
  if (scratch_for_current_device(&ds) != cudaSuccess) return NQPU_SIMULATION_FAILED;
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  double* sums = ds.addr + (kNoAllocScratchDoubles - kNoAllocSumSlots);  // n+1 <= 35 doubles at the end
  cudaError_t e = launch_zsums(dt, d_amplitudes, int(num_qubits), ds.addr, sums, st, ds.sms);
  if (e != cudaSuccess) return NQPU_SIMULATION_FAILED;
  k_z_from_sums<<<1, 64, 0, st>>>(sums, int(num_qubits), d_out);
  if (cudaGetLastError() != cudaSuccess) return NQPU_SIMULATION_FAILED;
  return NQPU_OK;
}
