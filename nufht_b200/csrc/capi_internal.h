// The opaque handle behind NufhtDevicePlan (include/nufht_b200.h), shared by the C-ABI
// translation units.
#pragma once

#include <memory>

#include "executor.h"

// Shared ownership: a batch (batch.cpp) keeps the plans it captured alive after the caller
// destroys the handle.
struct NufhtDevicePlan {
  std::shared_ptr<hankel::DevicePlan> dp;
};
