// Device implementation of the plan's level walk (plan_device.cu).
#pragma once

#include <memory>
#include <string>

#include <cuda_runtime.h>

#include "plan.hpp"

namespace dfb {

// The walker that runs the level walk on the current CUDA device; the same
// results as the host walk, bit for bit.
LevelWalker* device_level_walker();
// The octree build's particle ordering on the current CUDA device; the same
// cells and order as the host build, bit for bit.  One per prcmpt.
std::unique_ptr<TreeSorter> make_device_tree_sorter();
// The plan's FP64 transfer spectra (tables: tab_fund.size() x PP) and
// signatures (sig, sig2: the host layout, stages after each other) computed
// on the current device, bit-identical to the host's; 0 or -4 with err set.
int device_plan_tables(const Plan& p, double2* tables, double2* sig, double2* sig2, std::string& err);
// The near-field lists (Plan::nd) from the level walk's near pairs on the
// device (npair (target cell, source cell) pairs in walk order), with the
// host build's contents and order; also sets i_near and sym_scratch.
// 0, -4 (CUDA error) or -5 (out of device memory, or more than 2^31 ranges
// or scratch rows for the 32-bit sorts: the device walk then leaves the
// lists to the host build) with err set.
int device_near_lists(Plan& p, const int2* d_near, int64_t npair, std::string& err);
// FP64 -> FP32 complex, rounded to nearest.
void tables_to_float(const double2* in, float2* out, int64_t n, cudaStream_t s);

}  // namespace dfb
