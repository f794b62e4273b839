// Device implementation of the plan's level walk (plan_device.cu).
#pragma once

#include "plan.hpp"

namespace dfb {

// The walker that runs the level walk on the current CUDA device; the same
// results as the host walk, bit for bit.
LevelWalker* device_level_walker();

}  // namespace dfb
