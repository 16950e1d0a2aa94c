// The opaque plan object behind the C ABI's bfgt_plan handle.
#pragma once
#include "device_plan.hpp"
#include "host_plan.hpp"

#include <memory>
#include <utility>
#include <vector>

struct bfgt_plan_s {
  bfgt::HostPlan hp;
  bfgt::DevicePlan dp;
  double stage_ms[8] = {0};
  // [first, last) 0-based box ranges that hold every leaf box; the host-array
  // entry point moves only these (runs separated by a few non-leaf boxes are
  // merged, so a range may include some non-leaf boxes, which the transform
  // neither reads nor writes)
  std::vector<std::pair<int, int>> leaf_runs;
  // bytes the last host-array execute copied host to device (accumulator runs
  // that were all zero are cleared on the device instead)
  double last_h2d_bytes = 0, last_d2h_bytes = 0;
  // the transposed transform (bfgt_plan_execute_adjoint), built on first use
  std::unique_ptr<bfgt::HostPlan> adj_hp;
  std::unique_ptr<bfgt::DevicePlan> adj_dp;
};
