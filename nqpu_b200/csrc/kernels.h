// Launch wrappers of the sm_100a kernels, called by the host engine.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <vector>
#include "sv_types.h"

namespace nqpu {

// Arguments of a per-gate launch (passed by value).
struct PGArgs {
  uint64_t n_items;   // work items (index sets) of the launch
  uint64_t setmask;   // bits forced to one (controls)
  uint64_t cmask;     // controls checked per amplitude (elementwise kernels)
  int32_t npos;       // zero-bit insert positions, ascending
  int32_t pos[8];
  int32_t t0, t1;
  double m[32];
};

// --- per-gate path -----------------------------------------------------------
cudaError_t launch_pergate(DType dt, void* amp, int n, const Op& op, cudaStream_t s, int num_sms);

// --- tiled pass path ---------------------------------------------------------
int tile_kmax_for(DType dt);
// CTA configuration of the tiled pass kernel (1: one CTA/SM, double-buffered
// tiles; 2: two CTAs/SM, single-buffered).
void tile_config_set(DType dt, int minb);
int tile_config_get(DType dt);
cudaError_t launch_tile_pass(DType dt, void* amp, int n, const PassRec& host_pass,
                             const PassRec* d_passes, const StageRec* d_stages, const void* d_ops,
                             int pass_idx, cudaStream_t stream, int num_sms);

// --- state utilities ---------------------------------------------------------
cudaError_t launch_set_basis(DType dt, void* amp, int n, uint64_t index, cudaStream_t s, int num_sms);
cudaError_t launch_scale(DType dt, void* amp, int n, double factor, cudaStream_t s, int num_sms);
// zero amplitudes whose bit q differs from `keep`, scale the rest by `factor`
cudaError_t launch_collapse(DType dt, void* amp, int n, int q, int keep, double factor,
                            cudaStream_t s, int num_sms);
// |a_i|^2 for `count` amplitudes starting at `amp` (already offset by the caller).
cudaError_t launch_probabilities(DType dt, const void* amp, uint64_t count, double* out,
                                 cudaStream_t s, int num_sms);
// Convert `count` amplitudes between dtypes (either may equal the other).
cudaError_t launch_convert(DType src_dt, const void* src, DType dst_dt, void* dst, uint64_t count,
                           cudaStream_t s, int num_sms);

// --- FP64 reductions ---------------------------------------------------------
// Layout of the all-<Z_i> scratch (doubles): kZsMaxBlocks x kZsBlkVals
// per-block low-bit partials, then one total per segment of kZsSegVecs 128-bit
// vectors (room is kept for kZsSegSlots per segment).
constexpr int kZsBlkVals = 16;
constexpr int kZsMaxBlocks = 1024;
constexpr uint64_t kZsSegVecs = 256 * 16;  // threads per block x vectors per thread
constexpr int kZsSegSlots = 8;
// Doubles of all-<Z_i> scratch for a state of 2^vec_log2 128-bit vectors.
constexpr size_t zsums_scratch_doubles(int vec_log2) {
  return size_t(kZsMaxBlocks) * kZsBlkVals +
         size_t(((uint64_t(1) << vec_log2) + kZsSegVecs - 1) / kZsSegVecs) * kZsSegSlots;
}
// Scratch bytes every reduction below needs on an n-qubit state.
size_t reduce_scratch_bytes(int n);
// out[0] = sum |a|^2, out[1+q] = sum over amplitudes with bit q set of |a|^2, q < n.
cudaError_t launch_zsums(DType dt, const void* amp, int n, double* scratch, double* out,
                         cudaStream_t s, int num_sms);
// out[0..1] = sum conj(a) b (re, im)
cudaError_t launch_inner(DType dta, const void* a, DType dtb, const void* b, int n,
                         double* scratch, double* out, cudaStream_t s, int num_sms);
// Pauli-string expectation (R/lib.rs:465 semantics): xmask = X|Y positions,
// zmask = Z|Y positions, ny = number of Y factors.  out[0] = real part.
cudaError_t launch_pauli(DType dt, const void* amp, int n, uint64_t xmask, uint64_t zmask,
                         uint64_t ymask, double* scratch, double* out, cudaStream_t s,
                         int num_sms);
// Sampling with given uniforms: out[s] = first i with u[s] < cumsum_i, else 2^n-1.
cudaError_t launch_sample(DType dt, const void* amp, int n, const double* d_uniforms,
                          uint32_t shots, double* scratch, uint64_t* d_out, cudaStream_t s,
                          int num_sms);

}  // namespace nqpu
