// Batched execution of many circuits in one persistent launch (see
// kernels_batch.cu for the device side).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "sv_types.h"

namespace nqpu {

struct BatchCirc {
  uint64_t amp_off;    // first amplitude of the circuit's state in the HBM arena
  int32_t n;           // qubits
  int32_t small;       // 1: whole circuit in one CTA's shared memory
  int32_t pass_base;   // first PassRec of the circuit in the global pass table
  int32_t n_passes;
  int32_t done_base;   // first completion counter (n_passes pass counters + 1 measure counter)
  int32_t meas_tiles;  // measurement tiles (2^(n-13)); 0 for small circuits
  int32_t part_base;   // first per-tile <H> partial
  int32_t obs_base;    // J[0..n-2] then h[0..n-1] in the observable array
  int32_t result;      // output slot
  int32_t meas_k;      // measurement tile bits: min(13, n)
};

struct BatchTask {
  int32_t circ;
  int32_t phase;  // -1: whole small circuit; 0..n_passes-1: pass tile; n_passes: measure tile
  uint32_t tile;
  int32_t pad;
};

struct BatchLaunch {
  float* arena;
  const BatchCirc* circs;
  const BatchTask* tasks;
  uint32_t n_tasks;
  const PassRec* passes;
  const StageRec* stages;
  const TileOp<float>* ops;
  const double* obs;
  uint32_t* counters;
  double* partials;
  double* results;
  uint32_t* cursor;
  int* err;
  unsigned grid;
  uint32_t spin_limit;  // polls of a bounded dependency wait (0: kBatchSpinLimit)
};

// Default bound of a pass tile's dependency wait (polls of ~64 ns or more).
constexpr uint32_t kBatchSpinLimit = 1u << 26;

size_t batch_smem_bytes();
cudaError_t launch_batch(const BatchLaunch& L, cudaStream_t s);

}  // namespace nqpu
