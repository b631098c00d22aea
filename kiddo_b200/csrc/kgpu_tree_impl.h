// kgpu_tree_impl.h — definition of the opaque kgpu_tree handle, shared by the
// translation units that launch queries on it.
#pragma once

#include <mutex>

#include "../../include/kiddo_gpu.h"
#include "kgpu_launch.h"

struct kgpu_tree {
  kgpu::DeviceTree dt;
  std::mutex points_mu;  // guards the lazily built point table (kgpu_tree_project)
};

namespace kgpu {
// Validates a query description against a tree; `radius_family` selects the
// within/within().unsorted() families.  Returns a kgpu_status and records the
// message for kgpu_last_error().
int check_query_desc(const kgpu_tree* t, const kgpu_query_desc* d, bool radius_family);
// Whether nearest_n rows come out sorted (requested, or max_qty above the
// reference's unsorted ThresholdVec range of 24).
bool rows_sorted(const kgpu_query_desc* d);
// Whether a batch is processed grouped by leaf (KGPU_FLAG_[NO_]SPATIAL_ORDER).
bool want_spatial_order(uint32_t flags, uint64_t nq, uint64_t leaves);
// Copies the periodic box of `d` (if any) into the launch description.
void apply_periodic(const DeviceTree& dt, const kgpu_query_desc* d, QueryLaunch& q);
}  // namespace kgpu
