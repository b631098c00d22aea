// kgpu_chamfer.cu — Chamfer/ICP-style neighbour loss and its adjoint.
//
// Loss over source points s_i and their k nearest target points t_m (found by
// the nearest_n engine on the target tree, SquaredEuclidean, f32):
//     L = sum_i sum_{j < count_i} phi(d_ij),   d_ij = |t_m - s_i|^2,
//     phi(d) = d * exp(-d / (2 sigma^2))        (Gaussian-weighted squared distance)
// Adjoint, with phi'(d) = exp(-d / (2 sigma^2)) * (1 - d / (2 sigma^2)):
//     dL/ds_i = sum_j phi'(d_ij) * 2 (s_i - t_m)
//     dL/dt_m = - sum_{(i, j) : nbr_ij = m} phi'(d_ij) * 2 (s_i - t_m)
// Determinism without floating-point atomics: the loss is reduced in a fixed
// tree order; a source sums its neighbours in rank order; the (source,
// neighbour) pairs are bucketed by target with one stable radix sort of the
// pair ids on their target, so every bucket holds its pairs in pair-id order
// and is summed in that order (no atomics at all).
// d_ij is recomputed from the coordinates with the same rounded operations as
// the leaf scan ((0 + dx^2) + dy^2) + dz^2, so it equals the forward distance.
#include <cmath>
#include <cstdint>
#include <string>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "../../include/kiddo_gpu.h"
#include "kgpu_device.cuh"
#include "kgpu_devbuf.h"
#include "kgpu_internal.h"
#include "kgpu_launch.h"
#include "kgpu_tree_impl.h"

namespace kgpu {
namespace {


__device__ __forceinline__ float sq_dist3(const float* a, const float* b) {
  float acc = 0.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float t = __fsub_rn(a[d], b[d]);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
  }
  return acc;
}

// per-source loss: sum_j phi(d_ij) in rank order
__global__ void k_chamfer_loss(const float* __restrict__ dists, const uint32_t* __restrict__ counts,
                               uint64_t n_src, int k, float inv2s2, float* __restrict__ per_src) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n_src;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const int c = int(counts[i]);
    float acc = 0.f;
    for (int j = 0; j < c; ++j) {
      const float d = dists[i * k + j];
      acc += d * expf(-d * inv2s2);
    }
    per_src[i] = acc;
  }
}

// Fixed-order sum of n values: each block reduces a contiguous range in a fixed
// tree; a second launch with one block reduces the block sums the same way.
__global__ void k_fixed_sum(const float* __restrict__ x, uint64_t n, float* __restrict__ out) {
  __shared__ float sh[256];
  const uint64_t per = (n + gridDim.x - 1) / gridDim.x;
  const uint64_t lo = uint64_t(blockIdx.x) * per;
  const uint64_t hi = min(n, lo + per);
  float acc = 0.f;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) acc += x[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

__device__ __forceinline__ void load3(const float* p, uint64_t i, float (&v)[3]) {
  v[0] = p[i * 3 + 0];
  v[1] = p[i * 3 + 1];
  v[2] = p[i * 3 + 2];
}

// target index of neighbour (i, j): the item, offset by the pair's target base
__device__ __forceinline__ uint64_t target_of(const uint32_t* items, const uint32_t* tree_of,
                                              const uint64_t* tgt_base, uint64_t i, int k, int j) {
  const uint64_t base = tree_of ? tgt_base[tree_of[i]] : 0;
  return base + items[i * k + j];
}

__global__ void k_grad_src(const float* __restrict__ src, const float* __restrict__ tgt,
                           const uint32_t* __restrict__ items, const uint32_t* __restrict__ counts,
                           const uint32_t* __restrict__ tree_of, const uint64_t* __restrict__ tgt_base,
                           uint64_t n_src, int k, float inv2s2, float scale,
                           float* __restrict__ grad_src) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n_src;
       i += uint64_t(gridDim.x) * blockDim.x) {
    float s[3];
    load3(src, i, s);
    float g[3] = {0.f, 0.f, 0.f};
    const int c = int(counts[i]);
    for (int j = 0; j < c; ++j) {
      float t[3];
      load3(tgt, target_of(items, tree_of, tgt_base, i, k, j), t);
      const float d = sq_dist3(t, s);
      const float w = expf(-d * inv2s2) * (1.f - d * inv2s2) * 2.f;
#pragma unroll
      for (int a = 0; a < 3; ++a) g[a] += w * (s[a] - t[a]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) grad_src[i * 3 + a] = g[a] * scale;
  }
}

// Pair p = i * k + j (source i, rank j): its target when j < count_i, else
// n_tgt, which sorts after every real target.
__global__ void k_pair_keys(const uint32_t* __restrict__ items,
                            const uint32_t* __restrict__ counts,
                            const uint32_t* __restrict__ tree_of,
                            const uint64_t* __restrict__ tgt_base, uint64_t np, int k,
                            uint32_t n_tgt, uint32_t* __restrict__ key, uint32_t* __restrict__ id) {
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < np;
       p += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t i = p / uint32_t(k);
    const int j = int(p - i * uint32_t(k));
    key[p] = j < int(counts[i]) ? uint32_t(target_of(items, tree_of, tgt_base, i, k, j)) : n_tgt;
    id[p] = uint32_t(p);
  }
}

// start[m] = the first position of target m in the sorted keys, for m in
// 0..n_tgt (start[n_tgt] = the number of real pairs): each position a sets
// the targets after key[a - 1] up to key[a], and position np the rest.
__global__ void k_bucket_starts(const uint32_t* __restrict__ key, uint64_t np, uint64_t n_tgt,
                                uint64_t* __restrict__ start) {
  for (uint64_t a = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; a <= np;
       a += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t lo = a == 0 ? 0 : uint64_t(key[a - 1]) + 1;
    const uint64_t hi = a == np ? n_tgt : uint64_t(key[a]);
    for (uint64_t m = lo; m <= hi && m <= n_tgt; ++m) start[m] = a;
  }
}

// One target per thread: sum its pairs in pair-id order.
__global__ void k_grad_tgt(const float* __restrict__ src, const float* __restrict__ tgt,
                           const uint64_t* __restrict__ start, const uint32_t* __restrict__ pairs,
                           uint64_t n_tgt, int k, float inv2s2, float scale,
                           float* __restrict__ grad_tgt) {
  for (uint64_t m = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; m < n_tgt;
       m += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t lo = start[m], hi = start[m + 1];
    float t[3];
    load3(tgt, m, t);
    float g[3] = {0.f, 0.f, 0.f};
    for (uint64_t a = lo; a < hi; ++a) {
      const uint64_t i = pairs[a] / uint32_t(k);
      float s[3];
      load3(src, i, s);
      const float d = sq_dist3(t, s);
      const float w = expf(-d * inv2s2) * (1.f - d * inv2s2) * 2.f;
#pragma unroll
      for (int c = 0; c < 3; ++c) g[c] -= w * (s[c] - t[c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) grad_tgt[m * 3 + c] = g[c] * scale;
  }
}

int cuda_err(cudaError_t e, const char* what) {
  return set_error(KGPU_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int grid_of(uint64_t n) {
  const uint64_t b = (n + 255) / 256;
  const uint64_t cap = uint64_t(sm_count()) * 8;
  return int(b < cap ? (b ? b : 1) : cap);
}

}  // namespace
}  // namespace kgpu

using namespace kgpu;

extern "C" {

int32_t kgpu_chamfer_loss(const float* dists, const uint32_t* counts, uint64_t n_src, uint32_t k,
                          double sigma, float* per_src, float* loss, void* stream) {
  if (!dists || !counts || !loss || k == 0) return set_error(KGPU_EINVAL, "NULL argument or k == 0");
  if (!(sigma > 0)) return set_error(KGPU_EINVAL, "sigma must be positive");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DevBuf ps, part;
  float* per = per_src;
  cudaError_t e;
  if (!per) {
    if ((e = ps.alloc(n_src * 4, s)) != cudaSuccess) return set_error(KGPU_ENOMEM, "allocation");
    per = ps.as<float>();
  }
  const float inv2s2 = float(1.0 / (2.0 * sigma * sigma));
  if (n_src) {
    k_chamfer_loss<<<grid_of(n_src), 256, 0, s>>>(dists, counts, n_src, int(k), inv2s2, per);
    g_launches++;
  }
  const int nb = 512;
  if ((e = part.alloc(nb * 4, s)) != cudaSuccess) return set_error(KGPU_ENOMEM, "allocation");
  k_fixed_sum<<<nb, 256, 0, s>>>(per, n_src, part.as<float>());
  k_fixed_sum<<<1, 256, 0, s>>>(part.as<float>(), nb, loss);
  g_launches += 2;
  e = cudaGetLastError();
  return e == cudaSuccess ? KGPU_OK : cuda_err(e, "chamfer loss");
}

int32_t kgpu_chamfer_backward(const float* src, uint64_t n_src, const float* tgt, uint64_t n_tgt,
                              const uint32_t* items, const uint32_t* counts, uint32_t k,
                              const uint32_t* tree_of, const uint64_t* tgt_base, double sigma,
                              float grad_scale, float* grad_src, float* grad_tgt, void* stream) {
  if (!src || !tgt || !items || !counts || k == 0)
    return set_error(KGPU_EINVAL, "NULL argument or k == 0");
  if (!(sigma > 0)) return set_error(KGPU_EINVAL, "sigma must be positive");
  if ((tree_of == nullptr) != (tgt_base == nullptr))
    return set_error(KGPU_EINVAL, "tree_of and tgt_base go together");
  if (n_src * k >= (uint64_t(1) << 32)) return set_error(KGPU_EOVERFLOW, "n_src * k >= 2^32");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float inv2s2 = float(1.0 / (2.0 * sigma * sigma));
  cudaError_t e;
  if (grad_src && n_src) {
    k_grad_src<<<grid_of(n_src), 256, 0, s>>>(src, tgt, items, counts, tree_of, tgt_base, n_src,
                                              int(k), inv2s2, grad_scale, grad_src);
    g_launches++;
  }
  if (grad_tgt && n_tgt) {
    if (n_tgt >= 0xFFFFFFFFull) return set_error(KGPU_EOVERFLOW, "2^32 - 1 targets or more");
    DevBuf start, kin, vin, kout, vout, sort_tmp;
    const uint64_t np = n_src * k;
    int bits = 1;
    while (bits < 32 && (uint64_t(1) << bits) <= n_tgt) ++bits;
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, kin.as<uint32_t>(), kout.as<uint32_t>(),
                                    vin.as<uint32_t>(), vout.as<uint32_t>(), uint32_t(np), 0, bits,
                                    s);
    if ((e = start.alloc((n_tgt + 1) * 8, s)) != cudaSuccess ||
        (e = kin.alloc(np * 4, s)) != cudaSuccess || (e = vin.alloc(np * 4, s)) != cudaSuccess ||
        (e = kout.alloc(np * 4, s)) != cudaSuccess || (e = vout.alloc(np * 4, s)) != cudaSuccess ||
        (e = sort_tmp.alloc(sort_bytes, s)) != cudaSuccess)
      return set_error(KGPU_ENOMEM, "device allocation failed");
    if (np) {
      k_pair_keys<<<grid_of(np), 256, 0, s>>>(items, counts, tree_of, tgt_base, np, int(k),
                                             uint32_t(n_tgt), kin.as<uint32_t>(),
                                             vin.as<uint32_t>());
      g_launches++;
      if ((e = cub::DeviceRadixSort::SortPairs(sort_tmp.p, sort_bytes, kin.as<uint32_t>(),
                                               kout.as<uint32_t>(), vin.as<uint32_t>(),
                                               vout.as<uint32_t>(), uint32_t(np), 0, bits, s)) !=
          cudaSuccess)
        return cuda_err(e, "ordering the pairs");
    }
    k_bucket_starts<<<grid_of(np + 1), 256, 0, s>>>(kout.as<uint32_t>(), np, n_tgt,
                                                    start.as<uint64_t>());
    k_grad_tgt<<<grid_of(n_tgt), 256, 0, s>>>(src, tgt, start.as<uint64_t>(), vout.as<uint32_t>(),
                                              n_tgt, int(k), inv2s2, grad_scale, grad_tgt);
    g_launches += 2;
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? KGPU_OK : cuda_err(e, "chamfer backward");
}

}  // extern "C"
