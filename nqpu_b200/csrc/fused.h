// Fused execution mode: runs of gates packed into <=5-qubit unitaries applied
// as split-TF32 tensor-core contractions (tcgen05) over the statevector.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "sv_types.h"

namespace nqpu {
struct StateImpl;
bool fused_plan_build(const std::vector<Op>& ops, int n, DType dt, void** plan, PlanStats* stats);
bool fused_plan_stats(const std::vector<Op>& ops, int n, DType dt, PlanStats* stats);
void fused_plan_free(void* plan);
// Queue the plan's launches on the state's stream; its norm partials and
// bounded-wait flag live in the state's run scratch (state_run_error reads it).
cudaError_t fused_run(void* plan, StateImpl* s, std::vector<cudaEvent_t>* events);
}  // namespace nqpu
