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
cudaError_t fused_run(void* plan, StateImpl* s, std::vector<cudaEvent_t>* events);
// Reads the plan's device error flag (set when a bounded wait expired).
cudaError_t fused_check_error(void* plan, cudaStream_t st);
}  // namespace nqpu
