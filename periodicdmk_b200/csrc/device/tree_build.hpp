// Tree construction with the points on the GPU (tree_build.cu).
#pragma once
#include "../host/plan.hpp"

namespace pdmkb {

// build_plan with its point-heavy steps (lattice images, level-0 binning,
// octant partitions, Morton order inside the leaves) on the current CUDA
// device; the plan equals build_plan's.  Synchronous; throws as build_plan,
// and std::runtime_error ("CUDA error ...") on device failures.
Plan build_plan_device(const double* cell, int n, const double* pos, int n_digits, int n_per_leaf, int nz,
                       const double* bloch = nullptr);

// Where the library builds a tree of n points: on the device from
// min_device_points points up (the fixed costs of the device steps outweigh
// the host's point loops below it), unless PDMK_TREE_BUILD is "host" or
// "device".
bool tree_build_on_device(int n, int min_device_points);

}  // namespace pdmkb
