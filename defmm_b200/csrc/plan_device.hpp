// Device implementation of the plan's level walk (plan_device.cu).
#pragma once

#include <memory>

#include "plan.hpp"

namespace dfb {

// The walker that runs the level walk on the current CUDA device; the same
// results as the host walk, bit for bit.
LevelWalker* device_level_walker();
// The octree build's particle ordering on the current CUDA device; the same
// cells and order as the host build, bit for bit.  One per prcmpt.
std::unique_ptr<TreeSorter> make_device_tree_sorter();

}  // namespace dfb
