// kgpu_launch.h — host-side launch interface between the API and the kernels.
#pragma once

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/kiddo_gpu.h"

namespace kgpu {

struct DeviceTree {
  int dtype = 0;
  int dims = 0;
  int device = 0;
  void* stems = nullptr;       // A[stem_count]
  uint8_t* arena = nullptr;    // leaf bytes
  void* extents = nullptr;     // uint2 (offset/8, len) [leaf_count]
  int max_stem_level = -1;
  uint32_t leaf_count = 0;
  uint64_t size = 0;
  uint64_t stem_count = 0;
  uint64_t leaf_bytes_len = 0;
  uint64_t max_leaf_len = 0;
  size_t device_bytes = 0;
  uint32_t bh = 0;             // 0: Eytzinger stems; 3 or 4: Donnelly<bh>
  // Mapped stem/leaf resolution: u32 leaf of each stem index from map_min
  // (0xffffffff: not terminal) on the device, or null (arithmetic)
  uint32_t* leaf_map = nullptr;
  uint64_t map_min = 0;
  uint32_t map_len = 0;
  // the kernels' scalar backtracking walk (Donnelly stems or Mapped resolution)
  // rather than the Eytzinger arithmetic DFS
  bool scalar_walk() const { return bh != 0 || leaf_map != nullptr; }
  bool pooled = false;         // arrays from the stream-ordered pool (device-built trees)
  // f64 3-D leaves are 32-byte rows with offsets of their own: the reference
  // layout's extents, uint2 (offset / 8, len), for read-back; null otherwise
  void* src_extents = nullptr;
  // stored points of query results (kgpu_tree_project), built on first use:
  // the entries' points in iteration order, and (item, rank) sorted by item
  void* iter_points = nullptr;
  uint32_t* sorted_items = nullptr;
  uint32_t* sorted_ranks = nullptr;
  int items_distinct = -1;     // -1: not checked yet; 0: two entries share an item; 1: distinct
  // per-axis bounds of the stored points, measured on first use by periodic
  // queries (kgpu_periodic_fast.cu): -1 not measured, 0 unusable (no points,
  // or a NaN coordinate), 1 measured
  mutable int point_bounds = -1;
  mutable double point_lo[4] = {0, 0, 0, 0}, point_hi[4] = {0, 0, 0, 0};
};

struct QueryLaunch {
  int family = 0;     // kgpu_family
  int metric = 0;     // kgpu_metric
  int k = 1;
  double radius = 0;
  bool exclusive = false;
  bool sorted = true;
  const void* queries = nullptr;  // device, nq * dims values of A
  const uint32_t* order = nullptr;  // optional processing order (device)
  uint64_t nq = 0;
  void* out_d = nullptr;
  uint32_t* out_i = nullptr;
  uint32_t* out_c = nullptr;
  unsigned long long* stats = nullptr;  // optional [stems, leaves, points] totals
  uint32_t chunk = 64;            // queries handed to a warp at a time (lane-refilled drivers)
  int refill = 24;                // idle lanes a warp waits for before refilling them
  int engine = 0;                 // 0 auto, 1 warp per query, 2 thread per query,
                                  // 3 thread walks with warp-cooperative leaf scans
  bool periodic = false;          // periodic boundary conditions
  double box[4] = {0, 0, 0, 0};   // periodic box (converted to A)
  // batches over many trees (see kgpu_forest_*): device arrays, or null
  const void* forest = nullptr;          // TreeView<A>[n_trees]
  const uint32_t* tree_of = nullptr;     // tree of each query
  uint32_t n_trees = 0;
  const uint64_t* leaf_base = nullptr;   // first global leaf number of each tree
  uint64_t total_leaves = 0;             // leaves of all trees (spatial order)
  const void* radii = nullptr;           // per-query radius (A), or null
  unsigned long long* work = nullptr;    // work-queue counter (zeroed), or null
  const unsigned long long* nq_dev = nullptr;  // device count bounding nq (lane-refilled drivers)
  uint64_t capacity = ~uint64_t(0);      // fill pass: hits that fit the output
  int* status = nullptr;                 // fill pass: set to KGPU_EOVERFLOW on mismatch
  cudaStream_t stream = nullptr;
};

// process-wide count of kernel launches made by this library
extern std::atomic<uint64_t> g_launches;

// QueryLaunch::engine from a query's KGPU_FLAG_ENGINE_* bits.
inline int engine_of(uint32_t flags) {
  return (flags & KGPU_FLAG_ENGINE_WARP) ? 1 : (flags & KGPU_FLAG_ENGINE_THREAD) ? 2
         : (flags & KGPU_FLAG_ENGINE_COOP) ? 3 : 0;
}

// The launch knobs of kgpu_query_desc::tuning (KGPU_TUNE_*); 0 fields keep
// the defaults (24 idle lanes, 64-query chunks).
inline void apply_tuning(uint32_t tuning, QueryLaunch& q) {
  const uint32_t refill = tuning & 0x3fu;
  const uint32_t chunk_log2 = (tuning >> 8) & 0xfu;
  if (refill >= 1 && refill <= 32) q.refill = int(refill);
  if (chunk_log2 >= 5 && chunk_log2 <= 10) q.chunk = 1u << chunk_log2;
}

// Fixed-size families: dispatches to the thread engine (2-D/3-D trees) or the
// warp engine (everything else, periodic included).
template <typename A> cudaError_t launch_fixed(const DeviceTree& t, const QueryLaunch& q);

// Periodic sorted nearest_n over one tree through a plain walk where the box's
// faces cannot change a row, and the periodic walk for the other rows
// (kgpu_periodic_fast.cu).  `handled` is false, with nothing launched, where
// it does not apply; the caller then launches the periodic walk itself.
template <typename A>
cudaError_t periodic_fast(const DeviceTree& t, const QueryLaunch& q, bool& handled);
template <typename A> cudaError_t launch_wfixed(const DeviceTree& t, const QueryLaunch& q);
template <typename A> cudaError_t launch_tfixed(const DeviceTree& t, const QueryLaunch& q);
// Lists of any length held in the output rows (kernels_*_rows.cu).
template <typename A> cudaError_t launch_trow(const DeviceTree& t, const QueryLaunch& q);
// Donnelly-stem kernels, defined in their own translation units
// (kernels_f32_donnelly.cu, kernels_f64_donnelly.cu); the last argument only
// selects the coordinate type.
cudaError_t launch_tfixed_donnelly(const DeviceTree& t, const QueryLaunch& q, float);
cudaError_t launch_tfixed_donnelly(const DeviceTree& t, const QueryLaunch& q, double);
cudaError_t launch_within_donnelly(const DeviceTree& t, const QueryLaunch& q, uint64_t* counts,
                                   const uint64_t* offsets, float);
cudaError_t launch_within_donnelly(const DeviceTree& t, const QueryLaunch& q, uint64_t* counts,
                                   const uint64_t* offsets, double);
template <typename A> cudaError_t launch_within_count(const DeviceTree& t, const QueryLaunch& q,
                                                       uint64_t* counts);
template <typename A> cudaError_t launch_within_fill(const DeviceTree& t, const QueryLaunch& q,
                                                      const uint64_t* offsets);
// Processing order grouped by straight-descent leaf.  `scratch` must hold
// spatial_order_scratch_bytes(t, nq) bytes; order[nq] receives query indices.
size_t spatial_order_scratch_bytes(const DeviceTree& t, const QueryLaunch& q);
template <typename A> cudaError_t launch_spatial_order(const DeviceTree& t, const QueryLaunch& q,
                                                       uint32_t* order, void* scratch);

// Stable sort of every CSR segment by distance; scratch holds total entries.
// Segments are clamped to the first `capacity` entries.
template <typename A> cudaError_t launch_seg_sort(const uint64_t* offsets, uint64_t nq,
                                                  uint64_t capacity, A* d, uint32_t* it,
                                                  A* scratch_d, uint32_t* scratch_i,
                                                  cudaStream_t s);

// offsets[0..n] = exclusive prefix sum of counts[0..n) (offsets[n] = total).
// `counts` and `offsets` may alias.  tmp needs scan_tmp_bytes(n) bytes.
size_t scan_tmp_bytes(uint64_t n);
cudaError_t launch_exclusive_scan(const uint64_t* counts, uint64_t* offsets, uint64_t n,
                                  void* tmp, cudaStream_t s);

int sm_count();

// Re-encodes a tree's 3-D leaves between the reference's tiles (at the
// offsets of dt.src_extents, or of dt.extents when that is null) and the
// device's rows (at the offsets of dt.extents).
cudaError_t convert_leaf_layout(const DeviceTree& dt, const uint8_t* src, uint8_t* dst,
                                bool to_rows, cudaStream_t s);

}  // namespace kgpu
