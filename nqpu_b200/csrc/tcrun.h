// Tensor-core pass mode: device plans and their execution (tcpass.cu).
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "sv_types.h"
#include "tcpass.h"

namespace nqpu {
struct StateImpl;
// Plan (host, tcplan.cpp) and upload; false for complex128 or n < 12.
bool tc_plan_build(const std::vector<Op>& ops, int n, DType dt, void** plan, PlanStats* stats);
bool tc_plan_stats(const std::vector<Op>& ops, int n, DType dt, PlanStats* stats);
void tc_plan_free(void* plan);
// Queue every pass of the plan on the state's stream (one launch per pass).
cudaError_t tc_run(void* plan, StateImpl* s, std::vector<cudaEvent_t>* events);
// Queue the passes of a host plan whose records and B operands are already in
// device memory: pass i's record at d_passes + i, its B operands at d_bmats +
// bmat_off[i] (tc_bmat_offsets); d_norm holds 3 * slots doubles of scratch
// (the grid is at most `slots` CTAs), *d_err is set when a bounded wait
// expires.  With `events`, an event is recorded after every launch.
cudaError_t tc_launch(float* amp, const TcPlan& plan, const TcPassRec* d_passes, const uint16_t* d_bmats,
                      const size_t* bmat_off, double* d_norm, int slots, int* d_err, cudaStream_t st,
                      std::vector<cudaEvent_t>* events = nullptr);
void tc_bmat_offsets(const TcPlan& plan, std::vector<size_t>* off);
}  // namespace nqpu
