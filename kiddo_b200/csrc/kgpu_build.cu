// kgpu_build.cu — the ImmutableKdTree soft construction on the device.
//
// The same tree, byte for byte, as the host builder (layout_build.cpp, the
// reference's construction.rs:413-539, 868-968, 1089-1175), built level by
// level instead of recursively:
//
//  * every axis keeps the point ids sorted by that axis's coordinate (a stable
//    radix sort once, ties in id order), and every node owns the same segment
//    [begin, begin + len) of each axis's list;
//  * the nodes of a level split on axis level % K.  A node's ideal pivot is
//    ceil(len / 2) (soft_ideal_pivot with a power-of-two budget, clamped to
//    [1, len]); update_pivot's nudge is read off the sorted segment: lt = the
//    number of values below the ideal value v, le = the number not above it,
//    pivot = lt if lt > 0, else len if le == len (unsplittable, no stem),
//    else le.  The stem is the first value of the right part and the left part
//    is the first `pivot` ids of the segment, i.e. the points with a
//    coordinate below the stem;
//  * the other axes' lists are partitioned stably by that left / right side
//    with one prefix sum per axis, so each stays sorted inside every node;
//  * after the last level each leaf's points are sorted by source index and
//    written in the VecOfArenas tile encoding (leaf_strategy/vec_of_arenas.rs:
//    292-323), each leaf on an 8-byte boundary.
//
// One deliberate limit: a coordinate axis holding both -0.0 and +0.0 may give a
// stem of the other zero sign than the host builder's (which zero std's
// selection returns is unspecified); every other input gives the host's bytes.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <limits>
#include <new>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "../../include/kiddo_gpu.h"
#include "kgpu_devbuf.h"
#include "kgpu_device.cuh"
#include "kgpu_internal.h"
#include "kgpu_launch.h"
#include "kgpu_tree_impl.h"

namespace kgpu {
namespace {

constexpr uint32_t kBucket = 32;

template <typename A>
__global__ void k_fill(A* __restrict__ p, uint64_t n, A v) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x)
    p[i] = v;
}

template <typename A>
__global__ void k_axis_keys(const A* __restrict__ pts, uint64_t n, int K, int d,
                            A* __restrict__ keys, uint32_t* __restrict__ ids) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    keys[i] = pts[i * K + d];
    ids[i] = uint32_t(i);
  }
}

// One thread per node of the level: pivot, stem and left size.
template <typename A>
__global__ void k_split_level(const A* __restrict__ pts, int K, int d,
                              const uint32_t* __restrict__ perm, const uint64_t* __restrict__ nb,
                              const uint64_t* __restrict__ nl, uint64_t nodes, uint64_t stem_base,
                              A* __restrict__ stems, uint64_t* __restrict__ cut) {
  const uint64_t node = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (node >= nodes) return;
  const uint64_t b = nb[node], len = nl[node];
  uint64_t pivot = len;
  if (len > 0) {
    uint64_t ideal = (len + 1) / 2;
    if (ideal < 1) ideal = 1;
    if (ideal < len) {
      const A v = pts[uint64_t(perm[b + ideal]) * K + d];
      uint64_t lo = 0, hi = len;  // lt: first position whose value is not below v
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (pts[uint64_t(perm[b + mid]) * K + d] < v) lo = mid + 1;
        else hi = mid;
      }
      const uint64_t lt = lo;
      lo = lt;
      hi = len;  // le: first position whose value is above v
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (!(v < pts[uint64_t(perm[b + mid]) * K + d])) lo = mid + 1;
        else hi = mid;
      }
      const uint64_t le = lo;
      pivot = lt > 0 ? lt : (le >= len ? len : le);
    }
    if (pivot < len) stems[stem_base + node] = pts[uint64_t(perm[b + pivot]) * K + d];
  }
  cut[node] = pivot;
}

// side[id] = 1 for the points of the right part (positions of the split axis's list).
__global__ void k_mark_sides(const uint32_t* __restrict__ perm, uint64_t n,
                             const uint32_t* __restrict__ node_of, const uint64_t* __restrict__ nb,
                             const uint64_t* __restrict__ cut, uint8_t* __restrict__ side) {
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
       p += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t node = node_of[p];
    side[perm[p]] = (p - nb[node]) >= cut[node] ? 1 : 0;
  }
}

__global__ void k_left_flags(const uint32_t* __restrict__ perm, uint64_t n,
                             const uint8_t* __restrict__ side, uint64_t* __restrict__ flags) {
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
       p += uint64_t(gridDim.x) * blockDim.x)
    flags[p] = side[perm[p]] ? 0u : 1u;
}

// Stable partition of every node's segment: left ids first, both halves in
// their current order.  excl = exclusive prefix sum of the left flags.
__global__ void k_partition(const uint32_t* __restrict__ perm, uint64_t n,
                            const uint32_t* __restrict__ node_of, const uint64_t* __restrict__ nb,
                            const uint64_t* __restrict__ cut, const uint64_t* __restrict__ excl,
                            const uint8_t* __restrict__ side, uint32_t* __restrict__ out) {
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
       p += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t node = node_of[p];
    const uint64_t b = nb[node];
    const uint64_t lrank = excl[p] - excl[b];
    const uint32_t id = perm[p];
    out[side[id] ? b + cut[node] + ((p - b) - lrank) : b + lrank] = id;
  }
}

__global__ void k_next_nodes(uint64_t nodes, const uint64_t* __restrict__ nb,
                             const uint64_t* __restrict__ nl, const uint64_t* __restrict__ cut,
                             uint64_t* __restrict__ nb2, uint64_t* __restrict__ nl2) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nodes) return;
  nb2[2 * i] = nb[i];
  nl2[2 * i] = cut[i];
  nb2[2 * i + 1] = nb[i] + cut[i];
  nl2[2 * i + 1] = nl[i] - cut[i];
}

__global__ void k_next_node_of(uint64_t n, uint32_t* __restrict__ node_of,
                               const uint64_t* __restrict__ nb, const uint64_t* __restrict__ cut) {
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
       p += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t node = node_of[p];
    node_of[p] = 2u * node + ((p - nb[node]) >= cut[node] ? 1u : 0u);
  }
}

// Leaf sizes: id keys for the sort by source index, encoded bytes rounded up
// to 8 for the arena offsets, and the longest leaf.
template <typename A>
__global__ void k_leaf_sizes(const uint32_t* __restrict__ perm, uint64_t n, int K,
                             const uint64_t* __restrict__ nl, uint64_t leaves,
                             double* __restrict__ keys, uint32_t* __restrict__ ids,
                             uint64_t* __restrict__ bytes, unsigned long long* __restrict__ maxlen) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n || i < leaves;
       i += uint64_t(gridDim.x) * blockDim.x) {
    if (i < n) {
      keys[i] = double(perm[i]);
      ids[i] = perm[i];
    }
    if (i < leaves) {
      uint64_t len = nl[i], total = 0;
      while (len) {
        const uint64_t w = len >= 32 ? 32 : len >= 8 ? 8 : len >= 4 ? 4 : len >= 2 ? 2 : 1;
        total += w * (K * sizeof(A) + sizeof(uint32_t));
        len -= w;
      }
      bytes[i] = (total + 7) & ~uint64_t(7);
      atomicMax(maxlen, (unsigned long long)nl[i]);
    }
  }
}

// One warp per leaf: lane j writes point j's coordinates and item into its
// tile slot; extents as (offset / 8, len).
template <typename A, int K>
__global__ void k_write_leaves(const A* __restrict__ pts, const uint32_t* __restrict__ items,
                               const uint32_t* __restrict__ sorted_ids,
                               const uint64_t* __restrict__ nb, const uint64_t* __restrict__ nl,
                               const uint64_t* __restrict__ off, uint64_t leaves,
                               uint8_t* __restrict__ arena, uint2* __restrict__ extents,
                               uint2* __restrict__ src_extents) {
  const int lane = threadIdx.x & 31;
  for (uint64_t l = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; l < leaves;
       l += (uint64_t(gridDim.x) * blockDim.x) >> 5) {
    const uint64_t b = nb[l], len = nl[l];
    // f64 rows sit at 32 bytes per point before them; other leaves at the
    // reference's offsets
    const uint64_t o = src_extents ? b * row_bytes<A>() : off[l];
    if (lane == 0) {
      extents[l] = make_uint2(uint32_t(o / 8), uint32_t(len));
      if (src_extents) src_extents[l] = make_uint2(uint32_t(off[l] / 8), uint32_t(len));
    }
    uint8_t* leaf = arena + o;
    for (uint64_t p = lane; p < len; p += 32) {
      const uint32_t id = sorted_ids[b + p];
      uint32_t toff, w, i;
      tile_slot<A, K>(uint32_t(len), uint32_t(p), toff, w, i);
      A* col = reinterpret_cast<A*>(leaf + toff);
#pragma unroll
      for (int d = 0; d < K; ++d) col[d * w + i] = pts[uint64_t(id) * K + d];
      reinterpret_cast<uint32_t*>(leaf + toff + K * w * sizeof(A))[i] = items ? items[id] : id;
    }
  }
}

// Tiles <-> rows for the 3-D leaves held as rows on the device (RowLeaves),
// one warp per leaf: tiles at the reference's offsets (tex), rows at the
// device's (rex), the same point order.
template <typename A>
__device__ __forceinline__ void put_row(uint8_t* rows, uint32_t p, A x, A y, A z, uint32_t it) {
  if constexpr (sizeof(A) == 4) {
    reinterpret_cast<float4*>(rows)[p] = make_float4(x, y, z, __uint_as_float(it));
  } else {
    double2* r = reinterpret_cast<double2*>(rows) + 2 * size_t(p);
    r[0] = make_double2(x, y);
    r[1] = make_double2(z, __longlong_as_double((long long)it));  // item, then 4 zero bytes
  }
}

template <typename A>
__global__ void k_leaf_tiles_to_rows(const uint8_t* __restrict__ tiles, uint8_t* __restrict__ rows,
                                     const uint2* __restrict__ tex, const uint2* __restrict__ rex,
                                     uint64_t leaves) {
  const int lane = threadIdx.x & 31;
  for (uint64_t l = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; l < leaves;
       l += (uint64_t(gridDim.x) * blockDim.x) >> 5) {
    const uint2 te = tex[l];
    const size_t to = size_t(te.x) * 8, ro = size_t(rex[l].x) * 8;
    for (uint32_t p = lane; p < te.y; p += 32) {
      uint32_t toff, w, i;
      tile_slot_cols<A, 3>(te.y, p, toff, w, i);
      const A* col = reinterpret_cast<const A*>(tiles + to + toff);
      const uint32_t it = reinterpret_cast<const uint32_t*>(tiles + to + toff + 3 * w * sizeof(A))[i];
      put_row<A>(rows + ro, p, col[i], col[w + i], col[2 * w + i], it);
    }
  }
}

template <typename A>
__global__ void k_leaf_rows_to_tiles(const uint8_t* __restrict__ rows, uint8_t* __restrict__ tiles,
                                     const uint2* __restrict__ tex, const uint2* __restrict__ rex,
                                     uint64_t leaves) {
  const int lane = threadIdx.x & 31;
  for (uint64_t l = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; l < leaves;
       l += (uint64_t(gridDim.x) * blockDim.x) >> 5) {
    const uint2 te = tex[l];
    const size_t to = size_t(te.x) * 8, ro = size_t(rex[l].x) * 8;
    for (uint32_t p = lane; p < te.y; p += 32) {
      uint32_t toff, w, i;
      tile_slot_cols<A, 3>(te.y, p, toff, w, i);
      A c[3];
      uint32_t it;
      load_row<A, 3>(rows + ro, p, c, it);
      A* col = reinterpret_cast<A*>(tiles + to + toff);
      col[i] = c[0];
      col[w + i] = c[1];
      col[2 * w + i] = c[2];
      reinterpret_cast<uint32_t*>(tiles + to + toff + 3 * w * sizeof(A))[i] = it;
    }
  }
}

inline unsigned blocks_for(uint64_t n, unsigned threads = 256) {
  const uint64_t b = (n + threads - 1) / threads;
  return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 64)));
}

int cuda_fail_b(cudaError_t e, const char* what) {
  return set_error(e == cudaErrorMemoryAllocation ? KGPU_ENOMEM : KGPU_ECUDA,
                   std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename A, int K>
int build_on_device(const A* pts, const uint32_t* items, uint64_t n, cudaStream_t s,
                    DeviceTree& dt) {
  cudaError_t e;
  const uint64_t leaf_node_count = (n + kBucket - 1) / kBucket;
  uint32_t depth = 0;
  if (leaf_node_count >= 2)
    while ((uint64_t(1) << depth) < leaf_node_count) ++depth;
  const uint64_t leaves = n == 0 ? 0 : (uint64_t(1) << depth);
  const uint64_t stem_count = depth ? ((uint64_t(1) << (depth + 1)) + 7) / 8 * 8 : 0;
  dt.dtype = sizeof(A) == 8 ? KGPU_F64 : KGPU_F32;
  dt.dims = K;
  cudaGetDevice(&dt.device);
  dt.max_stem_level = depth ? int(depth) - 1 : -1;
  dt.leaf_count = uint32_t(leaves);
  dt.size = n;
  dt.stem_count = stem_count;
  dt.bh = 0;

  // per-axis id lists sorted by coordinate (stable, ties in id order)
  std::vector<DevBuf> perm(K);
  DevBuf keys_in, keys_out, ids_in, cub_tmp;
  if ((e = keys_in.alloc(n * sizeof(A), s)) != cudaSuccess ||
      (e = keys_out.alloc(n * sizeof(A), s)) != cudaSuccess ||
      (e = ids_in.alloc(n * 4, s)) != cudaSuccess)
    return cuda_fail_b(e, "construction scratch");
  size_t cub_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, keys_in.as<A>(), keys_out.as<A>(),
                                  ids_in.as<uint32_t>(), ids_in.as<uint32_t>(), int(n), 0,
                                  int(sizeof(A) * 8), s);
  if ((e = cub_tmp.alloc(cub_bytes, s)) != cudaSuccess) return cuda_fail_b(e, "sort scratch");
  for (int d = 0; d < K; ++d) {
    if ((e = perm[d].alloc(n * 4, s)) != cudaSuccess) return cuda_fail_b(e, "axis lists");
    if (n == 0) continue;
    k_axis_keys<A><<<blocks_for(n), 256, 0, s>>>(pts, n, K, d, keys_in.as<A>(),
                                                 ids_in.as<uint32_t>());
    g_launches++;
    size_t bytes = cub_bytes;
    if ((e = cub::DeviceRadixSort::SortPairs(cub_tmp.p, bytes, keys_in.as<A>(), keys_out.as<A>(),
                                             ids_in.as<uint32_t>(), perm[d].as<uint32_t>(),
                                             int(n), 0, int(sizeof(A) * 8), s)) != cudaSuccess)
      return cuda_fail_b(e, "sorting an axis");
  }

  // stems (+inf = no split); the tree's arrays come from the stream-ordered
  // pool, so rebuilding a tree of similar size reuses cached memory
  dt.pooled = true;
  if ((e = scratch_alloc(&dt.stems, std::max<size_t>(16, stem_count * sizeof(A)), s)) !=
      cudaSuccess)
    return cuda_fail_b(e, "stems");
  if (stem_count) {
    k_fill<A><<<blocks_for(stem_count), 256, 0, s>>>(static_cast<A*>(dt.stems), stem_count,
                                                     std::numeric_limits<A>::infinity());
    g_launches++;
  }

  // levels
  DevBuf nb, nl, nb2, nl2, cut, node_of, side, flags, excl, scan_tmp, tmp_perm;
  const uint64_t maxnodes = std::max<uint64_t>(leaves, 1);
  if ((e = nb.alloc(maxnodes * 8, s)) != cudaSuccess || (e = nl.alloc(maxnodes * 8, s)) != cudaSuccess ||
      (e = nb2.alloc(maxnodes * 8, s)) != cudaSuccess || (e = nl2.alloc(maxnodes * 8, s)) != cudaSuccess ||
      (e = cut.alloc(maxnodes * 8, s)) != cudaSuccess || (e = node_of.alloc(n * 4, s)) != cudaSuccess ||
      (e = side.alloc(n, s)) != cudaSuccess || (e = flags.alloc((n + 1) * 8, s)) != cudaSuccess ||
      (e = excl.alloc((n + 1) * 8, s)) != cudaSuccess ||
      (e = scan_tmp.alloc(scan_tmp_bytes(n + 1), s)) != cudaSuccess ||
      (e = tmp_perm.alloc(n * 4, s)) != cudaSuccess)
    return cuda_fail_b(e, "construction scratch");
  const uint64_t zero = 0;
  if ((e = cudaMemcpyAsync(nb.p, &zero, 8, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(nl.p, &n, 8, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(node_of.p, 0, n * 4, s)) != cudaSuccess)
    return cuda_fail_b(e, "construction set-up");
  for (uint32_t level = 0; level < depth; ++level) {
    const uint64_t nodes = uint64_t(1) << level;
    const int d = int(level % K);
    k_split_level<A><<<blocks_for(nodes), 256, 0, s>>>(
        pts, K, d, perm[d].as<uint32_t>(), nb.as<uint64_t>(), nl.as<uint64_t>(), nodes, nodes,
        static_cast<A*>(dt.stems), cut.as<uint64_t>());
    k_mark_sides<<<blocks_for(n), 256, 0, s>>>(perm[d].as<uint32_t>(), n, node_of.as<uint32_t>(),
                                               nb.as<uint64_t>(), cut.as<uint64_t>(),
                                               side.as<uint8_t>());
    g_launches += 2;
    for (int a = 0; a < K; ++a) {
      if (a == d) continue;  // the split axis's list is already partitioned
      k_left_flags<<<blocks_for(n), 256, 0, s>>>(perm[a].as<uint32_t>(), n, side.as<uint8_t>(),
                                                 flags.as<uint64_t>());
      g_launches++;
      if ((e = launch_exclusive_scan(flags.as<uint64_t>(), excl.as<uint64_t>(), n, scan_tmp.p,
                                     s)) != cudaSuccess)
        return cuda_fail_b(e, "partition scan");
      k_partition<<<blocks_for(n), 256, 0, s>>>(perm[a].as<uint32_t>(), n, node_of.as<uint32_t>(),
                                                nb.as<uint64_t>(), cut.as<uint64_t>(),
                                                excl.as<uint64_t>(), side.as<uint8_t>(),
                                                tmp_perm.as<uint32_t>());
      g_launches++;
      std::swap(perm[a].p, tmp_perm.p);
    }
    k_next_nodes<<<blocks_for(nodes), 256, 0, s>>>(nodes, nb.as<uint64_t>(), nl.as<uint64_t>(),
                                                   cut.as<uint64_t>(), nb2.as<uint64_t>(),
                                                   nl2.as<uint64_t>());
    k_next_node_of<<<blocks_for(n), 256, 0, s>>>(n, node_of.as<uint32_t>(), nb.as<uint64_t>(),
                                                 cut.as<uint64_t>());
    g_launches += 2;
    std::swap(nb.p, nb2.p);
    std::swap(nl.p, nl2.p);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail_b(e, "construction levels");

  // leaves: ids by source index, sizes, offsets, arena
  DevBuf lkeys, lids, sk, si, lbytes, loff, lmax;
  if ((e = lkeys.alloc(n * 8, s)) != cudaSuccess || (e = lids.alloc(n * 4, s)) != cudaSuccess ||
      (e = sk.alloc(n * 8, s)) != cudaSuccess || (e = si.alloc(n * 4, s)) != cudaSuccess ||
      (e = lbytes.alloc((leaves + 1) * 8, s)) != cudaSuccess ||
      (e = loff.alloc((leaves + 1) * 8, s)) != cudaSuccess ||
      (e = lmax.alloc(8, s)) != cudaSuccess)
    return cuda_fail_b(e, "leaf scratch");
  if ((e = cudaMemsetAsync(lmax.p, 0, 8, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(lbytes.p, 0, (leaves + 1) * 8, s)) != cudaSuccess)
    return cuda_fail_b(e, "leaf set-up");
  uint64_t max_leaf = 0, arena_bytes = 0;
  if (leaves) {
    k_leaf_sizes<A><<<blocks_for(std::max(n, leaves)), 256, 0, s>>>(
        perm[0].as<uint32_t>(), n, K, nl.as<uint64_t>(), leaves, lkeys.as<double>(),
        lids.as<uint32_t>(), lbytes.as<uint64_t>(), lmax.as<unsigned long long>());
    g_launches++;
    // segment offsets of the leaves = their begins, plus n at the end
    DevBuf seg;
    if ((e = seg.alloc((leaves + 1) * 8, s)) != cudaSuccess) return cuda_fail_b(e, "leaf offsets");
    if ((e = cudaMemcpyAsync(seg.p, nb.p, leaves * 8, cudaMemcpyDeviceToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(seg.as<uint64_t>() + leaves, &n, 8, cudaMemcpyHostToDevice, s)) !=
            cudaSuccess)
      return cuda_fail_b(e, "leaf offsets");
    if ((e = launch_exclusive_scan(lbytes.as<uint64_t>(), loff.as<uint64_t>(), leaves + 1,
                                   scan_tmp.p, s)) != cudaSuccess)
      return cuda_fail_b(e, "arena offsets");
    if ((e = cudaMemcpyAsync(&max_leaf, lmax.p, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&arena_bytes, loff.as<uint64_t>() + leaves, 8,
                             cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return cuda_fail_b(e, "leaf sizes");
    if (max_leaf > 1024)
      return set_error(KGPU_EOVERFLOW,
                       "a leaf holds more than 1024 points (leaf scratch capacity, "
                       "leaf_view/mod.rs:18,58-65)");
    // sort every leaf's ids by source index (exact as double keys)
    if ((e = launch_seg_sort<double>(seg.as<uint64_t>(), leaves, n, lkeys.as<double>(),
                                     lids.as<uint32_t>(), sk.as<double>(), si.as<uint32_t>(), s)) !=
        cudaSuccess)
      return cuda_fail_b(e, "sorting the leaves");
    // the last leaf's bytes were counted rounded up to 8; the host arena ends at
    // the encoded end of the last leaf
    uint64_t last_len = 0;
    if ((e = cudaMemcpyAsync(&last_len, nl.as<uint64_t>() + leaves - 1, 8, cudaMemcpyDeviceToHost,
                             s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return cuda_fail_b(e, "leaf sizes");
    uint64_t raw = 0, rem = last_len;
    while (rem) {
      const uint64_t w = rem >= 32 ? 32 : rem >= 8 ? 8 : rem >= 4 ? 4 : rem >= 2 ? 2 : 1;
      raw += w * (K * sizeof(A) + sizeof(uint32_t));
      rem -= w;
    }
    arena_bytes = arena_bytes - ((raw + 7) & ~uint64_t(7)) + raw;
  }
  dt.leaf_bytes_len = arena_bytes;
  // f64 3-D rows: 32 bytes per point, offsets of their own
  const bool moved = RowLeaves<A, K>::value && sizeof(A) == 8;
  const uint64_t dev_bytes = moved ? n * row_bytes<A>() : arena_bytes;
  dt.max_leaf_len = max_leaf;
  if ((e = scratch_alloc(reinterpret_cast<void**>(&dt.arena), std::max<size_t>(16, dev_bytes + 16),
                         s)) != cudaSuccess ||
      (e = scratch_alloc(&dt.extents, std::max<size_t>(16, leaves * 8), s)) != cudaSuccess ||
      (moved && (e = scratch_alloc(&dt.src_extents, std::max<size_t>(16, leaves * 8), s)) !=
                    cudaSuccess))
    return cuda_fail_b(e, "tree arrays");
  if ((e = cudaMemsetAsync(dt.arena, 0, dev_bytes + 16, s)) != cudaSuccess)
    return cuda_fail_b(e, "arena");
  if (leaves) {
    k_write_leaves<A, K><<<blocks_for(leaves * 32), 256, 0, s>>>(
        pts, items, lids.as<uint32_t>(), nb.as<uint64_t>(), nl.as<uint64_t>(), loff.as<uint64_t>(),
        leaves, dt.arena, static_cast<uint2*>(dt.extents),
        static_cast<uint2*>(dt.src_extents));
    g_launches++;
  }
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return cuda_fail_b(e, "writing the leaves");
  dt.device_bytes = std::max<size_t>(16, stem_count * sizeof(A)) + dev_bytes + 16 +
                    leaves * 8 * (moved ? 2 : 1);
  return KGPU_OK;
}

}  // namespace

cudaError_t convert_leaf_layout(const DeviceTree& dt, const uint8_t* src, uint8_t* dst,
                                bool to_rows, cudaStream_t s) {
  if (dt.leaf_count == 0) return cudaSuccess;
  const unsigned grid = blocks_for(uint64_t(dt.leaf_count) * 32);
  const uint2* rex = static_cast<const uint2*>(dt.extents);
  const uint2* tex = dt.src_extents ? static_cast<const uint2*>(dt.src_extents) : rex;
  if (dt.dtype == KGPU_F64) {
    if (to_rows) k_leaf_tiles_to_rows<double><<<grid, 256, 0, s>>>(src, dst, tex, rex, dt.leaf_count);
    else k_leaf_rows_to_tiles<double><<<grid, 256, 0, s>>>(src, dst, tex, rex, dt.leaf_count);
  } else {
    if (to_rows) k_leaf_tiles_to_rows<float><<<grid, 256, 0, s>>>(src, dst, tex, rex, dt.leaf_count);
    else k_leaf_rows_to_tiles<float><<<grid, 256, 0, s>>>(src, dst, tex, rex, dt.leaf_count);
  }
  g_launches++;
  return cudaGetLastError();
}

namespace {

template <typename A>
int build_any_dims(int K, const void* pts, const uint32_t* items, uint64_t n, cudaStream_t s,
                   DeviceTree& dt) {
  const A* p = static_cast<const A*>(pts);
  switch (K) {
    case 1: return build_on_device<A, 1>(p, items, n, s, dt);
    case 2: return build_on_device<A, 2>(p, items, n, s, dt);
    case 3: return build_on_device<A, 3>(p, items, n, s, dt);
    case 4: return build_on_device<A, 4>(p, items, n, s, dt);
  }
  return set_error(KGPU_EUNSUPPORTED, "dims must be 1..4");
}

}  // namespace
}  // namespace kgpu

using namespace kgpu;

extern "C" {

int32_t kgpu_tree_build(int32_t dtype, uint32_t dims, const void* points, const uint32_t* items,
                        uint64_t n, void* stream, kgpu_tree** out) {
  if (!out) return set_error(KGPU_EINVAL, "out is NULL");
  *out = nullptr;
  if (dims < 1 || dims > uint32_t(kMaxDims)) return set_error(KGPU_EUNSUPPORTED, "dims must be 1..4");
  if (dtype != KGPU_F32 && dtype != KGPU_F64)
    return set_error(KGPU_EINVAL, "dtype must be KGPU_F32 or KGPU_F64");
  if (n > 0 && !points) return set_error(KGPU_EINVAL, "points is NULL");
  if (n >= (uint64_t(1) << 31)) return set_error(KGPU_EOVERFLOW, "2^31 points or more");
  auto* t = new (std::nothrow) kgpu_tree();
  if (!t) return set_error(KGPU_ENOMEM, "host allocation failed");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int st = dtype == KGPU_F64
                     ? build_any_dims<double>(int(dims), points, items, n, s, t->dt)
                     : build_any_dims<float>(int(dims), points, items, n, s, t->dt);
  if (st != KGPU_OK) {
    cudaStreamSynchronize(s);
    release_tree_arrays(t->dt);
    delete t;
    return st;
  }
  *out = t;
  return KGPU_OK;
}

int32_t kgpu_tree_read_layout(const kgpu_tree* t, void* stems, uint8_t* leaf_bytes,
                              uint64_t* extents, void* stream) {
  if (!t) return set_error(KGPU_EINVAL, "NULL tree");
  const DeviceTree& dt = t->dt;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t sa = dt.dtype == KGPU_F64 ? 8 : 4;
  std::vector<uint32_t> ex(2 * size_t(dt.leaf_count));
  cudaError_t e;
  // leaves held as rows go back to the reference's tiles first
  DevBuf tiles;
  const uint8_t* arena = dt.arena;
  if (leaf_bytes && dt.leaf_bytes_len && dt.dims == 3) {
    if ((e = tiles.alloc(dt.leaf_bytes_len, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(tiles.p, 0, dt.leaf_bytes_len, s)) != cudaSuccess ||
        (e = convert_leaf_layout(dt, dt.arena, tiles.as<uint8_t>(), false, s)) != cudaSuccess)
      return cuda_fail_b(e, "reading the layout");
    arena = tiles.as<uint8_t>();
  }
  if ((stems && dt.stem_count &&
       (e = cudaMemcpyAsync(stems, dt.stems, dt.stem_count * sa, cudaMemcpyDeviceToHost, s)) !=
           cudaSuccess) ||
      (leaf_bytes && dt.leaf_bytes_len &&
       (e = cudaMemcpyAsync(leaf_bytes, arena, dt.leaf_bytes_len, cudaMemcpyDeviceToHost, s)) !=
           cudaSuccess) ||
      (dt.leaf_count &&
       (e = cudaMemcpyAsync(ex.data(), dt.src_extents ? dt.src_extents : dt.extents,
                            ex.size() * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess))
    return cuda_fail_b(e, "reading the layout");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail_b(e, "reading the layout");
  if (extents)
    for (size_t l = 0; l < dt.leaf_count; ++l) {
      extents[2 * l] = uint64_t(ex[2 * l]) * 8;
      extents[2 * l + 1] = ex[2 * l + 1];
    }
  return KGPU_OK;
}

}  // extern "C"
