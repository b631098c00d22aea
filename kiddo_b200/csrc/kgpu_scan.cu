// kgpu_scan.cu — exclusive prefix sum of per-query hit counts (u64) that turns
// the counting pass of a radius query into CSR offsets.
//
// Three kernels: per-tile totals, a single-block scan of the tile totals, and
// a per-tile scan that adds the tile's base.  Each tile is 256 threads x 8
// consecutive counts, so the counts are read twice and the offsets written
// once: 24 bytes of HBM traffic per query.
#include <cstdint>
#include <cuda_runtime.h>

#include "kgpu_launch.h"

namespace kgpu {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr uint64_t kTile = uint64_t(kThreads) * kItems;

__device__ __forceinline__ uint64_t warp_incl_scan(uint64_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ uint64_t block_excl_scan(uint64_t v, uint64_t& excl) {
  __shared__ uint64_t warp_tot[kThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint64_t inc = warp_incl_scan(v);
  if (lane == 31) warp_tot[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint64_t t = lane < kThreads / 32 ? warp_tot[lane] : 0;
    const uint64_t ti = warp_incl_scan(t);
    if (lane < kThreads / 32) warp_tot[lane] = ti - t;  // exclusive warp bases
  }
  __syncthreads();
  excl = warp_tot[wid] + inc - v;
  __shared__ uint64_t block_total;
  if (threadIdx.x == kThreads - 1) block_total = excl + v;
  __syncthreads();
  const uint64_t bt = block_total;
  __syncthreads();
  return bt;
}

__global__ void __launch_bounds__(kThreads) k_tile_totals(const uint64_t* __restrict__ counts,
                                                          uint64_t n, uint64_t* __restrict__ tiles) {
  const uint64_t base = uint64_t(blockIdx.x) * kTile + uint64_t(threadIdx.x) * kItems;
  uint64_t s = 0;
#pragma unroll
  for (int j = 0; j < kItems; ++j)
    if (base + j < n) s += counts[base + j];
  uint64_t excl;
  const uint64_t tot = block_excl_scan(s, excl);
  if (threadIdx.x == 0) tiles[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kThreads) k_scan_tiles(uint64_t* __restrict__ tiles,
                                                         uint64_t ntiles) {
  uint64_t carry = 0;
  for (uint64_t b = 0; b < ntiles; b += kThreads) {
    const uint64_t i = b + threadIdx.x;
    const uint64_t v = i < ntiles ? tiles[i] : 0;
    uint64_t excl;
    const uint64_t tot = block_excl_scan(v, excl);
    if (i < ntiles) tiles[i] = carry + excl;
    carry += tot;
  }
  if (threadIdx.x == 0) tiles[ntiles] = carry;
}

__global__ void __launch_bounds__(kThreads) k_tile_apply(const uint64_t* counts, uint64_t n,
                                                         const uint64_t* __restrict__ tiles,
                                                         uint64_t ntiles, uint64_t* offsets) {
  const uint64_t base = uint64_t(blockIdx.x) * kTile + uint64_t(threadIdx.x) * kItems;
  uint64_t v[kItems];
  uint64_t s = 0;
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    v[j] = base + j < n ? counts[base + j] : 0;
    s += v[j];
  }
  uint64_t excl;
  block_excl_scan(s, excl);  // contains __syncthreads: all reads are done before writes
  uint64_t run = tiles[blockIdx.x] + excl;
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    if (base + j < n) offsets[base + j] = run;
    run += v[j];
  }
  if (blockIdx.x == ntiles - 1 && threadIdx.x == 0) offsets[n] = tiles[ntiles];
}

}  // namespace

size_t scan_tmp_bytes(uint64_t n) { return size_t((n + kTile - 1) / kTile + 1) * sizeof(uint64_t); }

size_t spatial_order_scratch_bytes(const DeviceTree& t, const QueryLaunch& q) {
  const uint64_t nl = q.forest ? q.total_leaves : (t.leaf_count > 0 ? t.leaf_count : 1);
  return ((q.nq * 4 + 255) / 256) * 256 + (((nl + 1) * 8 + 255) / 256) * 256 +
         scan_tmp_bytes(nl) + 256;
}

cudaError_t launch_exclusive_scan(const uint64_t* counts, uint64_t* offsets, uint64_t n, void* tmp,
                                  cudaStream_t s) {
  uint64_t* tiles = static_cast<uint64_t*>(tmp);
  if (n == 0) {
    cudaError_t e = cudaMemsetAsync(offsets, 0, sizeof(uint64_t), s);
    return e;
  }
  const uint64_t ntiles = (n + kTile - 1) / kTile;
  k_tile_totals<<<unsigned(ntiles), kThreads, 0, s>>>(counts, n, tiles);
  k_scan_tiles<<<1, kThreads, 0, s>>>(tiles, ntiles);
  k_tile_apply<<<unsigned(ntiles), kThreads, 0, s>>>(counts, n, tiles, ntiles, offsets);
  g_launches += 3;
  return cudaGetLastError();
}

}  // namespace kgpu
