// Tensor-core pass mode: device plans and their execution (tcpass.cu).
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "sv_types.h"

namespace nqpu {
struct StateImpl;
// Plan (host, tcplan.cpp) and upload; false for complex128 or n < 12.
bool tc_plan_build(const std::vector<Op>& ops, int n, DType dt, void** plan, PlanStats* stats);
bool tc_plan_stats(const std::vector<Op>& ops, int n, DType dt, PlanStats* stats);
void tc_plan_free(void* plan);
// Queue every pass of the plan on the state's stream (one launch per pass).
cudaError_t tc_run(void* plan, StateImpl* s, std::vector<cudaEvent_t>* events);
// Reads the plan's device error flag (set when a bounded wait expired).
cudaError_t tc_check_error(void* plan, cudaStream_t st);
}  // namespace nqpu
