// Split-precision (tensor-core) plane-wave kernels.
#include "../../include/bfgt.h"
#include "split_kernels.cuh"

namespace bfgt {

int split_plan_create(DevicePlan &, const HostPlan &, std::string &msg) {
  msg = "split precision is not built in this library";
  return BFGT_ERR_ARG;
}
void split_form(DevicePlan &, const double *, cudaStream_t) {}
void split_eval(DevicePlan &, double *, cudaStream_t) {}

}  // namespace bfgt
