// A batch of plans (independent trees, deltas, orders and densities) whose
// transforms run together: one launch per stage and kernel variant for all
// the plans' work, driven by device-side work lists of (plan, item) pairs.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <string>
#include <vector>

#include "device_plan.hpp"
#include "split_kernels.cuh"

namespace bfgt {

struct DeviceBatch {
  std::vector<DevicePlan *> plans;   // not owned
  std::vector<long long> offs;       // nplans + 1 element offsets of the packed fvals/pot
  SplitBatch split;                  // form/eval work of the split-precision plans
  void *tr_descs = nullptr, *nf_descs = nullptr;  // per-plan arguments (device)
  int2 *tr_work = nullptr, *nf_work = nullptr;    // {plan, block of the plan}
  int tr_blocks = 0, nf_blocks = 0;
  size_t smem_near = 0;
  // block near-field kernels: per-plan arguments, {plan, CTA} work of the
  // order-8 and order-16 plans on the tensor cores (0, 1) and in FP64 (2, 3)
  void *ntc_descs = nullptr;
  int2 *ntc_work[4] = {nullptr, nullptr, nullptr, nullptr};
  int ntc_blocks[4] = {0, 0, 0, 0};
  size_t smem_ntc[4] = {0, 0, 0, 0};
  std::vector<std::array<cudaEvent_t, 6>> evsets;
  int nrec = 0;
  bool events = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
};

int device_batch_create(DeviceBatch &b, const std::vector<DevicePlan *> &plans, std::string &msg);
// Queues the transforms of every plan on stream: fvals/pot are the packed
// arrays (plan i at element offset offs[i]).  FP64 plans run their form and
// eval stages as launches of their own; everything else is shared.
int device_batch_execute(DeviceBatch &b, const double *d_fvals, double *d_pot, cudaStream_t s, std::string &msg);
int device_batch_launches(const DeviceBatch &b);
int device_batch_stage_ms(DeviceBatch &b, double *out);
void device_batch_destroy(DeviceBatch &b);

int reserve_event_sets(std::vector<std::array<cudaEvent_t, 6>> &evsets, int n);
int read_stage_ms(std::vector<std::array<cudaEvent_t, 6>> &evsets, int &nrec, double *out);

}  // namespace bfgt
