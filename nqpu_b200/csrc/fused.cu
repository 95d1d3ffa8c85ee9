#include "fused.h"
#include "engine.h"
namespace nqpu {
bool fused_plan_build(const std::vector<Op>&, int, DType, void** plan, PlanStats*) { *plan = nullptr; return false; }
bool fused_plan_stats(const std::vector<Op>&, int, DType, PlanStats*) { return false; }
void fused_plan_free(void*) {}
cudaError_t fused_run(void*, StateImpl*, std::vector<cudaEvent_t>*) { return cudaErrorNotSupported; }
}  // namespace nqpu
