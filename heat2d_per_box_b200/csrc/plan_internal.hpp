// The opaque plan object behind the C ABI's bfgt_plan handle.
#pragma once
#include "device_plan.hpp"
#include "host_plan.hpp"

struct bfgt_plan_s {
  bfgt::HostPlan hp;
  bfgt::DevicePlan dp;
  double stage_ms[8] = {0};
};
