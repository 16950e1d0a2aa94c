// Split-precision (tensor-core) variants of the plane-wave kernels.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "device_plan.hpp"
#include "fgt_common.cuh"

namespace bfgt {

ReduceArgs reduce_args(const DevicePlan &dp);

// Uploads the BF16 operand slices of the level tables; BFGT_* status.
int split_plan_create(DevicePlan &dp, const HostPlan &hp, std::string &msg);
// leaf values -> partial cutoff expansions (same output as k_form_fp64)
void split_form(DevicePlan &dp, const double *d_fvals, cudaStream_t s);
// cutoff expansions -> leaf values, accumulated into pot (same as k_eval_fp64)
void split_eval(DevicePlan &dp, double *d_pot, cudaStream_t s);
void split_plan_destroy(DevicePlan &dp);
// Times the plan's compiled shape choices on its own work lists (scratch
// arrays; synchronous) and keeps the fastest: form with Y as float2 or
// double2 and 1 or 2 x-contraction tiles per thread, eval with step groups of
// 8, 4 or 2 on the chunks or their column halves.  Every choice gives the
// same bits.  report: best form and eval
// ms per launch, and the numbers of choices timed.
int split_autotune(DevicePlan &dp, cudaStream_t s, double *report, std::string &msg);

// Work lists of a batch of plans whose form and eval stages run as one launch
// per kernel variant (all chunks of all split plans in the batch).
struct SplitBatch {
  struct Group {
    int variant, begin, count;
    size_t smem;
  };
  void *form_descs = nullptr, *eval_descs = nullptr;  // per-plan kernel arguments (device)
  int2 *form_work = nullptr, *eval_work = nullptr;     // {plan, chunk}, grouped by variant
  std::vector<Group> form_groups, eval_groups;
};
// offs[i]: element offset of plan i's arrays in the packed fvals/pot
int split_batch_create(SplitBatch &b, const std::vector<DevicePlan *> &plans, const std::vector<long long> &offs,
                       std::string &msg);
void split_batch_form(const SplitBatch &b, const double *fbase, cudaStream_t s);
void split_batch_eval(const SplitBatch &b, double *pbase, cudaStream_t s);
int split_batch_launches(const SplitBatch &b);
void split_batch_destroy(SplitBatch &b);
// Reads and clears the device error flag of the tensor-core kernels (waits
// for the device); BFGT_ERR_TIMEOUT if a bounded wait gave up.
int split_check(DevicePlan &dp);
// Poll limit of every bounded mbarrier wait unless a plan sets its own.
unsigned int split_default_wait_iters();

}  // namespace bfgt
