// Engine objects behind the C ABI handles: device context, device-resident
// states and circuits with their cached execution plans.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "../../include/nqpu_b200.h"
#include "planner.h"
#include "sv_types.h"

namespace nqpu {

double next_random_f64();

// Device context: device_ready() is true when a CUDA device exists; work runs
// on the caller's current device, and device_sms() is that device's SM count.
bool device_ready();
int device_sms();

struct StateImpl {
  uint32_t n = 0;
  DType dt = DType::C128;
  void* amp = nullptr;         // 2^n amplitudes in HBM
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  double* scratch = nullptr;   // reduction scratch (reduce_scratch_bytes)
  double* d_small = nullptr;   // small device outputs (256 doubles)
  double* h_small = nullptr;   // pinned host mirror of d_small
  double* d_uni = nullptr;     // sampling uniforms
  uint64_t* d_shots = nullptr; // sampling outcomes
  uint32_t shot_cap = 0;
  // scratch of the tensor and fused passes (per state, so one circuit run on
  // two states whose streams overlap does not share it): per-CTA norm
  // partials and the bounded-wait expiry flag
  double* run_norm = nullptr;
  size_t run_norm_cap = 0;     // doubles
  int* run_err = nullptr;
};

StateImpl* state_new(uint32_t n, DType dt);
void state_free(StateImpl* s);
// The state's run scratch with room for `doubles` norm partials (grown on
// demand), its expiry flag cleared on the state's stream.
cudaError_t state_run_scratch(StateImpl* s, size_t doubles, double** norm, int** err);
// cudaErrorLaunchTimeout when the last tensor / fused run's bounded wait
// expired (synchronises the state's stream).
cudaError_t state_run_error(StateImpl* s);
// out (n+1 values): [0] = sum|a|^2, [1+q] = sum over bit q set; either pointer may be null.
cudaError_t state_zsums(const StateImpl* s, double* zs, double* total);
cudaError_t state_pauli(const StateImpl* s, uint64_t xm, uint64_t zm, uint64_t ym, double* out2);
cudaError_t state_inner(const StateImpl* a, const StateImpl* b, double* out2);
cudaError_t state_sample(const StateImpl* s, const double* uniforms, uint32_t shots, uint64_t* out);
cudaError_t state_probabilities(const StateImpl* s, double* out);
cudaError_t state_download_c128(const StateImpl* s, NqpuComplex* out);
cudaError_t state_upload_c128(StateImpl* s, const NqpuComplex* in);

// Cached device plan of a circuit for one (state size, dtype, mode).
struct DevicePlan {
  uint64_t version = ~0ull;
  TilePlan tile;
  std::vector<Op> ops;         // lowered ops (per-gate mode)
  PassRec* d_passes = nullptr;
  StageRec* d_stages = nullptr;
  void* d_ops = nullptr;
  void* fused = nullptr;       // fused-mode plan (owned by the fused module)
  void* tc = nullptr;          // tensor-core pass plan (owned by tcpass.cu)
  int kmax = 0;                // tile bits the tiled plan was built for
  PlanStats stats;
};

struct CircuitImpl {
  uint32_t n = 0;
  std::vector<GateRec> gates;
  uint64_t version = 0;
  // cached plans per (state qubits, dtype, mode, segment); segments are the
  // gate runs between mid-circuit measurements / resets
  std::map<std::tuple<uint32_t, int, int, int>, DevicePlan*> plans;
  // NQPU_MODE_AUTO's choice per (state qubits, dtype, segment): (circuit
  // version + 1, mode); version + 1 so that a default entry reads as unset
  std::map<std::tuple<uint32_t, int, int>, std::pair<uint64_t, int>> auto_modes;
  std::mutex mu;
};

// Gate runs of a circuit between mid-circuit measure / reset gates:
// [begin, end) ranges of c->gates, with the mid gate that follows (index, or
// -1 after the last run).
struct Segment {
  size_t begin, end;
  long mid;
};
std::vector<Segment> circuit_segments(const std::vector<GateRec>& gates);
bool circuit_has_mid(const std::vector<GateRec>& gates);
// Append gates given as the flat arrays of nqpu_circuit_add_gates (each
// checked as its single add would check it; nothing is appended unless all
// are valid).  Defined with the C ABI (capi.cpp).
NqpuError circuit_append_gates(CircuitImpl* c, const uint32_t* codes, const int32_t* qubits, const double* params,
                               const NqpuComplex* matrices, size_t count);

// Measure one qubit (collapse with the thread-local RNG draw, c_ffi.rs:537-560
// rule) / project it onto |0> and renormalise (lib.rs:1705).
cudaError_t state_measure(StateImpl* s, uint32_t qubit, uint32_t* outcome, double* probability);
cudaError_t state_reset_qubit(StateImpl* s, uint32_t qubit);

void circuit_free(CircuitImpl* c);
// Queue the circuit on the state's stream (no host sync).  With `events`, an
// event is recorded before the first launch and after every launch.
cudaError_t circuit_run(CircuitImpl* c, StateImpl* s, int mode,
                        std::vector<cudaEvent_t>* events = nullptr,
                        std::vector<uint32_t>* outcomes = nullptr);
bool circuit_plan_stats(const CircuitImpl* c, uint32_t n, DType dt, int mode, PlanStats* out);
// The mode NQPU_MODE_AUTO runs a lowered gate run in on an n-qubit state.
int auto_mode_for(const std::vector<Op>& ops, uint32_t n, DType dt);

// Run a lowered op list on a state with the given mode (used by batch/server).
cudaError_t run_ops_pergate(StateImpl* s, const std::vector<Op>& ops);

}  // namespace nqpu
