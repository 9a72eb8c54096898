// The opaque handle behind NufhtDevicePlan (include/nufht_b200.h), shared by the C-ABI
// translation units.
#pragma once

#include <memory>

#include "executor.h"

struct NufhtDevicePlan {
  std::unique_ptr<hankel::DevicePlan> dp;
};
