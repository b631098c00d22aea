// kgpu_internal.h — host-side internals shared by the library's translation units.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/kiddo_gpu.h"

namespace kgpu {

constexpr int kMaxDims = 4;
constexpr int kMaxK = 32;          // largest max_qty served by the register top-k lists
constexpr int kMaxBigK = 256;      // largest nearest_n k (shared-memory lists, warp engine)
constexpr int kMaxRowK = 1 << 20;  // largest k with the lists in the output rows
constexpr int kMaxThreadK = 64;    // largest nearest_n k on the thread engine (128-thread blocks)
constexpr int kMaxStemLevel = 30;  // 31 levels: one continuation slot per lane, u32 stem index

// Host copy of a tree layout as the reference stores it.
struct Layout {
  int dtype = 0;
  int dims = 0;
  uint64_t size = 0;
  int32_t max_stem_level = -1;
  uint64_t max_leaf_len = 0;
  uint32_t block_height = 0;         // 0: Eytzinger stems; 3 or 4: Donnelly<block_height>
  std::vector<uint8_t> stems_bytes;  // stem_count * sizeof(A)
  std::vector<uint8_t> leaf_bytes;
  std::vector<uint64_t> extents;     // (offset, len) pairs
};

// A process-unique id of the calling thread's current CUDA context (cuCtxGetId),
// or 0 if there is none.  It changes when a context is destroyed and made
// again (cudaDeviceReset), which invalidates device addresses cached per
// device.
uint64_t current_context_id();

// Records `msg` as the calling thread's last error and returns `status`.
int set_error(int status, const std::string& msg);

int build_layout_any(Layout& L, int dtype, int K, const void* pts, const uint32_t* items,
                     uint64_t n, int nthreads, uint32_t block_height = 0);

// The VecOfArenas arena and byte extents of a FlatVec tree's leaves: K point
// columns, items and (start, end) extents in points.
int flatvec_to_layout(Layout& L, int dtype, int K, const void* const* columns,
                      const uint32_t* items, const uint32_t* extents, uint64_t leaf_count,
                      uint64_t size);

}  // namespace kgpu

struct kgpu_layout {
  kgpu::Layout L;
};
