// kgpu_points.cu — a tree's entries in iteration order, and the stored points
// of query results.
//
// The reference iterates a tree leaf by leaf, leaf 0 to leaf_count - 1, each
// leaf's entries in stored order (KdTreeIter, src/kd_tree/iter.rs:54-90); an
// entry's position in that sequence is its rank here.  Its point projection
// (QueryBuilder::with_points, src/kd_tree/query/builder.rs:1982-1987) reads
// the hits' coordinates from the same sequence (builder.rs:2175-2305).
//
//  * kgpu_tree_iter writes the sequence: one warp per leaf, each lane one
//    entry, at the leaf's first rank (an exclusive scan of the leaf lengths).
//  * kgpu_tree_project maps result items back to their entries.  On its first
//    call for a tree it builds the tree's table: the points in rank order, and
//    the (item, rank) pairs sorted by item (one radix sort); it checks that no
//    two entries share an item, since only then does an item name one entry.
//    Each result item is then found by binary search in the table.
#include <cstdint>
#include <mutex>
#include <string>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "../../include/kiddo_gpu.h"
#include "kgpu_devbuf.h"
#include "kgpu_device.cuh"
#include "kgpu_internal.h"
#include "kgpu_launch.h"
#include "kgpu_launch_impl.cuh"
#include "kgpu_tree_impl.h"

namespace kgpu {
namespace {

constexpr uint32_t kNoRank = 0xFFFFFFFFu;

int points_grid(uint64_t threads) {
  const uint64_t b = (threads + 255) / 256;
  const uint64_t cap = uint64_t(sm_count()) * 8;
  return int(b < cap ? (b ? b : 1) : cap);
}

int cuda_fail(cudaError_t e, const char* what) {
  return set_error(KGPU_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

__global__ void k_leaf_lens(const uint2* __restrict__ extents, uint32_t leaf_count,
                            uint64_t* __restrict__ lens) {
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < leaf_count;
       l += gridDim.x * blockDim.x)
    lens[l] = extents[l].y;
}

// Entry p of leaf l goes to rank starts[l] + p.
template <typename A, int K>
__global__ void k_iter_entries(TreeView<A> tv, const uint64_t* __restrict__ starts,
                               uint32_t* __restrict__ items, A* __restrict__ pts) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t l = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; l < tv.leaf_count;
       l += nwarps) {
    const uint2 ex = tv.extents[l];
    const uint8_t* leaf = tv.arena + uint64_t(ex.x) * 8;
    const uint64_t base = starts[l];
    for (uint32_t p = lane; p < ex.y; p += 32) {
      A c[K];
      uint32_t it;
      load_point<A, K>(leaf, ex.y, p, c, it);
      if (items) items[base + p] = it;
      if (pts) {
#pragma unroll
        for (int d = 0; d < K; ++d) pts[(base + p) * K + d] = c[d];
      }
    }
  }
}

__global__ void k_iota(uint32_t* __restrict__ r, uint64_t n) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x)
    r[i] = uint32_t(i);
}

__global__ void k_shared_items(const uint32_t* __restrict__ sorted, uint64_t n,
                               int* __restrict__ flag) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i + 1 < n;
       i += uint64_t(gridDim.x) * blockDim.x)
    if (sorted[i] == sorted[i + 1]) *flag = 1;
}

// Rank and point of each item; kNoRank and zeros for an item not in the tree
// (the 0xFFFFFFFF of an unused result slot included, unless it is an item).
template <typename A>
__global__ void k_project(const uint32_t* __restrict__ items, uint64_t n,
                          const uint32_t* __restrict__ sitems,
                          const uint32_t* __restrict__ sranks, uint64_t size,
                          const A* __restrict__ ipts, int K, uint32_t* __restrict__ out_ranks,
                          A* __restrict__ out_pts) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t it = items[i];
    uint64_t lo = 0, hi = size;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (sitems[mid] < it) lo = mid + 1;
      else hi = mid;
    }
    const bool found = lo < size && sitems[lo] == it;
    const uint32_t r = found ? sranks[lo] : kNoRank;
    if (out_ranks) out_ranks[i] = r;
    if (out_pts)
      for (int d = 0; d < K; ++d) out_pts[i * K + d] = found ? ipts[uint64_t(r) * K + d] : A(0);
  }
}

// First rank of every leaf: starts[leaf_count] (device, caller-owned).
int leaf_starts(const DeviceTree& t, uint64_t* starts, cudaStream_t s) {
  const uint32_t L = t.leaf_count;
  DevBuf lens, tmp;
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, static_cast<uint64_t*>(nullptr), starts, L,
                                s);
  cudaError_t e;
  if ((e = lens.alloc(size_t(L) * 8, s)) != cudaSuccess ||
      (e = tmp.alloc(tmp_bytes, s)) != cudaSuccess)
    return set_error(KGPU_ENOMEM, "device allocation failed");
  k_leaf_lens<<<points_grid(L), 256, 0, s>>>(static_cast<const uint2*>(t.extents), L,
                                            lens.as<uint64_t>());
  g_launches++;
  if ((e = cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, lens.as<uint64_t>(), starts, L, s)) !=
      cudaSuccess)
    return cuda_fail(e, "scanning the leaf lengths");
  return KGPU_OK;
}

template <typename A>
int iter_entries(const DeviceTree& t, uint32_t* items, A* pts, cudaStream_t s) {
  DevBuf starts;
  if (starts.alloc(size_t(t.leaf_count) * 8, s) != cudaSuccess)
    return set_error(KGPU_ENOMEM, "device allocation failed");
  int st = leaf_starts(t, starts.as<uint64_t>(), s);
  if (st != KGPU_OK) return st;
  const TreeView<A> tv = make_view<A>(t);
  const int grid = points_grid(uint64_t(t.leaf_count) * 32);
  const uint64_t* sp = starts.as<uint64_t>();
  switch (t.dims) {
    case 1: k_iter_entries<A, 1><<<grid, 256, 0, s>>>(tv, sp, items, pts); break;
    case 2: k_iter_entries<A, 2><<<grid, 256, 0, s>>>(tv, sp, items, pts); break;
    case 3: k_iter_entries<A, 3><<<grid, 256, 0, s>>>(tv, sp, items, pts); break;
    case 4: k_iter_entries<A, 4><<<grid, 256, 0, s>>>(tv, sp, items, pts); break;
    default: return set_error(KGPU_EINVAL, "unsupported dimensionality");
  }
  g_launches++;
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? KGPU_OK : cuda_fail(e, "iterating the leaves");
}

int iter_any(const DeviceTree& t, uint32_t* items, void* pts, cudaStream_t s) {
  if (t.dtype == KGPU_F64) return iter_entries<double>(t, items, static_cast<double*>(pts), s);
  return iter_entries<float>(t, items, static_cast<float*>(pts), s);
}

// Builds the table of kgpu_tree_project once per tree (the caller holds the
// tree's lock).  Leaves dt.items_distinct at 1 with the table, or at 0.
int build_point_table(DeviceTree& t, cudaStream_t s) {
  const uint64_t n = t.size;
  const size_t esz = t.dtype == KGPU_F64 ? 8 : 4;
  DevBuf keys, vals, tmp, flag;
  size_t sort_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, static_cast<const uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr),
                                  static_cast<const uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), uint32_t(n), 0, 32, s);
  cudaError_t e;
  void* pts = nullptr;
  uint32_t* sitems = nullptr;
  uint32_t* sranks = nullptr;
  auto undo = [&](int st) {
    cudaFree(pts);
    cudaFree(sitems);
    cudaFree(sranks);
    return st;
  };
  if ((e = cudaMalloc(&pts, n * t.dims * esz)) != cudaSuccess ||
      (e = cudaMalloc(reinterpret_cast<void**>(&sitems), n * 4)) != cudaSuccess ||
      (e = cudaMalloc(reinterpret_cast<void**>(&sranks), n * 4)) != cudaSuccess ||
      (e = keys.alloc(n * 4, s)) != cudaSuccess || (e = vals.alloc(n * 4, s)) != cudaSuccess ||
      (e = tmp.alloc(sort_bytes, s)) != cudaSuccess || (e = flag.alloc(4, s)) != cudaSuccess)
    return undo(set_error(KGPU_ENOMEM, "device allocation failed"));
  int st = iter_any(t, keys.as<uint32_t>(), pts, s);
  if (st != KGPU_OK) return undo(st);
  k_iota<<<points_grid(n), 256, 0, s>>>(vals.as<uint32_t>(), n);
  g_launches++;
  if ((e = cub::DeviceRadixSort::SortPairs(tmp.p, sort_bytes, keys.as<uint32_t>(), sitems,
                                           vals.as<uint32_t>(), sranks, uint32_t(n), 0, 32,
                                           s)) != cudaSuccess)
    return undo(cuda_fail(e, "sorting the items"));
  int shared = 0;
  if ((e = cudaMemsetAsync(flag.p, 0, 4, s)) != cudaSuccess)
    return undo(cuda_fail(e, "checking the items"));
  k_shared_items<<<points_grid(n), 256, 0, s>>>(sitems, n, flag.as<int>());
  g_launches++;
  if ((e = cudaMemcpyAsync(&shared, flag.p, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return undo(cuda_fail(e, "checking the items"));
  if (shared) {
    t.items_distinct = 0;
    return undo(KGPU_OK);
  }
  t.iter_points = pts;
  t.sorted_items = sitems;
  t.sorted_ranks = sranks;
  t.items_distinct = 1;
  return KGPU_OK;
}

}  // namespace
}  // namespace kgpu

using namespace kgpu;

extern "C" {

int32_t kgpu_tree_iter(kgpu_tree* tree, uint32_t* out_items, void* out_points, void* stream) {
  if (!tree) return set_error(KGPU_EINVAL, "NULL tree");
  const DeviceTree& t = tree->dt;
  if (t.size == 0 || t.leaf_count == 0 || (!out_items && !out_points)) return KGPU_OK;
  return iter_any(t, out_items, out_points, static_cast<cudaStream_t>(stream));
}

int32_t kgpu_tree_project(kgpu_tree* tree, const uint32_t* items, uint64_t n, uint32_t* out_ranks,
                          void* out_points, void* stream) {
  if (!tree) return set_error(KGPU_EINVAL, "NULL tree");
  if (n && !items) return set_error(KGPU_EINVAL, "NULL items");
  DeviceTree& t = tree->dt;
  if (t.size >= kNoRank)
    return set_error(KGPU_EUNSUPPORTED,
                     "point projection takes trees of fewer than 2^32 - 1 entries");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  {
    std::lock_guard<std::mutex> lock(tree->points_mu);
    if (t.items_distinct < 0 && t.size) {
      const int st = build_point_table(t, s);
      if (st != KGPU_OK) return st;
    }
    if (t.items_distinct == 0)
      return set_error(KGPU_EUNSUPPORTED,
                       "point projection needs distinct items: two entries of this tree share one");
  }
  if (n == 0 || (!out_ranks && !out_points)) return KGPU_OK;
  const int grid = points_grid(n);
  if (t.dtype == KGPU_F64)
    k_project<double><<<grid, 256, 0, s>>>(items, n, t.sorted_items, t.sorted_ranks, t.size,
                                           static_cast<const double*>(t.iter_points), t.dims,
                                           out_ranks, static_cast<double*>(out_points));
  else
    k_project<float><<<grid, 256, 0, s>>>(items, n, t.sorted_items, t.sorted_ranks, t.size,
                                          static_cast<const float*>(t.iter_points), t.dims,
                                          out_ranks, static_cast<float*>(out_points));
  g_launches++;
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? KGPU_OK : cuda_fail(e, "projecting the results");
}

}  // extern "C"
