// kgpu_launch_impl.cuh — dispatch from runtime options to kernel instantiations.
#pragma once

#include <type_traits>

#include "../../include/kiddo_gpu.h"
#include "kgpu_internal.h"
#include "kgpu_kernels.cuh"
#include "kgpu_launch.h"

namespace kgpu {

template <typename A>
inline TreeView<A> make_view(const DeviceTree& t) {
  TreeView<A> v;
  v.stems = static_cast<const A*>(t.stems);
  v.arena = t.arena;
  v.extents = static_cast<const uint2*>(t.extents);
  v.max_stem_level = t.max_stem_level;
  v.leaf_count = t.leaf_count;
  v.size = t.size;
  v.stem_count = t.stem_count;
  v.bh = t.bh;
  v.leaf_map = t.leaf_map;
  v.map_min = t.map_min;
  v.map_len = t.map_len;
  return v;
}

// Persistent grid: as many blocks of `threads` threads as fit on all SMs at once.
template <typename Kern>
inline int grid_for(Kern kern, size_t smem, uint64_t work_warps, int threads = 256) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const uint64_t full = uint64_t(per_sm) * sm_count();
  const uint64_t warps = uint64_t(threads) / 32;
  const uint64_t need = (work_warps + warps - 1) / warps;
  return int(need < full ? (need > 0 ? need : 1) : full);
}

template <typename F>
inline cudaError_t with_dims(int dims, F&& f) {
  switch (dims) {
    case 1: return f(std::integral_constant<int, 1>());
    case 2: return f(std::integral_constant<int, 2>());
    case 3: return f(std::integral_constant<int, 3>());
    case 4: return f(std::integral_constant<int, 4>());
  }
  return cudaErrorInvalidValue;
}

template <typename F>
inline cudaError_t with_metric(int metric, F&& f) {
  if (metric == KGPU_MANHATTAN) return f(Manhattan());
  if (metric == KGPU_CHEBYSHEV) return f(Chebyshev());
  if (metric == KGPU_MINKOWSKI3) return f(Minkowski<3>());
  if (metric == KGPU_MINKOWSKI4) return f(Minkowski<4>());
  return f(SqEuclidean());
}

template <typename F>
inline cudaError_t with_excl(bool e, F&& f) {
  if (e) return f(std::true_type());
  return f(std::false_type());
}

template <typename A>
inline Batch<A> make_batch(const QueryLaunch& q) {
  Batch<A> b;
  b.Q = static_cast<const A*>(q.queries);
  b.order = q.order;
  b.nq = q.nq;
  b.forest = static_cast<const TreeView<A>*>(q.forest);
  b.tree_of = q.tree_of;
  b.n_trees = q.n_trees;
  b.radii = static_cast<const A*>(q.radii);
  b.work = q.work;
  b.chunk = q.chunk;
  b.refill = q.refill;
  b.nq_dev = q.nq_dev;
  return b;
}

template <typename A, int K>
inline BoxArg<A, K> make_box(const QueryLaunch& q) {
  BoxArg<A, K> box;
  for (int d = 0; d < K; ++d) box.v[d] = A(q.box[d]);
  return box;
}

// Dynamic shared memory of the thread-per-query kernels (one slot per level).
template <typename A>
inline size_t thread_smem(const DeviceTree& t) {
  return size_t(t.max_stem_level + 2) * 256 * sizeof(A);
}

// Dynamic shared memory of the periodic per-thread walks: the rd slots, for
// Donnelly stems a column of path stem indices, then 3K columns of cell state
// (bounds and offsets) per thread.
template <typename A>
inline size_t periodic_smem(const DeviceTree& t, int stems) {
  return thread_smem<A>(t) + (stems ? size_t(t.max_stem_level + 2) * 256 * sizeof(uint32_t) : 0) +
         size_t(3 * t.dims) * 256 * sizeof(A);
}

// 2-D and 3-D trees have thread-per-query kernels; other dimensionalities use
// the warp kernels (same results).
constexpr bool thread_engine_dims(int K) { return K == 2 || K == 3; }

template <typename A>
cudaError_t launch_wfixed(const DeviceTree& t, const QueryLaunch& q) {
  const TreeView<A> tv = make_view<A>(t);
  const Batch<A> b = make_batch<A>(q);
  const A radius = A(q.radius);
  return with_dims(t.dims, [&](auto kk) {
    constexpr int K = decltype(kk)::value;
    return with_metric(q.metric, [&](auto m) {
      using M = decltype(m);
      return with_excl(q.exclusive, [&](auto ex) {
        constexpr bool EX = decltype(ex)::value;
        if constexpr (!M::kPeriodic) {
          if (q.periodic) return cudaErrorInvalidValue;  // rejected by the entry points
        } else if (q.periodic) {
          const auto box = make_box<A, K>(q);
          auto runp = [&](auto kern) {
            const int grid = grid_for(kern, 0, q.nq);
            kern<<<grid, 256, 0, q.stream>>>(tv, b, box, q.k, radius, static_cast<A*>(q.out_d),
                                             q.out_i, q.out_c, q.stats);
            g_launches++;
            return cudaGetLastError();
          };
          if (q.family == KGPU_NEAREST_ONE)
            return runp(k_periodic_fixed<A, K, M, KF_NEAREST_ONE, false>);
          if (q.family == KGPU_NEAREST_N || q.family == KGPU_NEAREST_N_WITHIN)
            return runp(k_periodic_fixed<A, K, M, KF_NEAREST_N, EX>);
          return cudaErrorInvalidValue;
        }
        auto run = [&](auto kern) {
          const int grid = grid_for(kern, 0, q.nq);
          kern<<<grid, 256, 0, q.stream>>>(tv, b, q.k, radius, q.sorted ? 0 : 1,
                                           static_cast<A*>(q.out_d), q.out_i, q.out_c, q.stats);
          g_launches++;
          return cudaGetLastError();
        };
        switch (q.family) {
          case KGPU_NEAREST_ONE:
            return run(k_fixed<A, K, M, KF_NEAREST_ONE, false>);
          case KGPU_APPROX_NEAREST_ONE:
            return run(k_fixed<A, K, M, KF_APPROX, false>);
          case KGPU_NEAREST_N:
          case KGPU_NEAREST_N_WITHIN:
            if (q.k > kMaxK) {
              const size_t smem = size_t(8) * q.k * (sizeof(A) + 8);
              auto kern = k_fixed_bign<A, K, M, KF_NEAREST_N, EX>;
              cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
              const int grid = grid_for(kern, smem, q.nq);
              kern<<<grid, 256, smem, q.stream>>>(tv, b, q.k, radius, q.sorted ? 0 : 1,
                                                  static_cast<A*>(q.out_d), q.out_i, q.out_c,
                                                  q.stats);
              g_launches++;
              return cudaGetLastError();
            }
            return run(k_fixed<A, K, M, KF_NEAREST_N, EX>);
          case KGPU_BEST_N_WITHIN:
            if (q.k > kMaxK) {
              const size_t smem = size_t(8) * q.k * (sizeof(A) + 8);
              auto kern = k_fixed_bign<A, K, M, KF_BEST_N, EX>;
              cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
              const int grid = grid_for(kern, smem, q.nq);
              kern<<<grid, 256, smem, q.stream>>>(tv, b, q.k, radius, 0, static_cast<A*>(q.out_d),
                                                  q.out_i, q.out_c, q.stats);
              g_launches++;
              return cudaGetLastError();
            }
            return run(k_fixed<A, K, M, KF_BEST_N, EX>);
        }
        return cudaErrorInvalidValue;
      });
    });
  });
}

// Thread-per-query fixed-size families.  Only 2-D and 3-D trees; the caller
// checks.  Shared memory per block: continuation slots plus, for the list
// families, k (distance, item) pairs per thread.
// STEMS: 0 for Eytzinger stems (arithmetic DFS), 1 for Donnelly stems
// (scalar backtracking); the Donnelly instantiation lives in its own
// translation units (kernels_*_donnelly.cu).
template <typename A, int STEMS>
cudaError_t launch_tfixed_stems(const DeviceTree& t, const QueryLaunch& q) {
  const TreeView<A> tv = make_view<A>(t);
  const Batch<A> b = make_batch<A>(q);
  const A radius = A(q.radius);
  const int levels = t.max_stem_level + 2;
  const bool list = q.family == KGPU_NEAREST_N || q.family == KGPU_NEAREST_N_WITHIN ||
                    q.family == KGPU_BEST_N_WITHIN;
  // nearest_n lists of 33..kMaxThreadK entries fit in shared memory with
  // 128-thread blocks (at k = 64: 64 KB of lists per block, 96 KB in f64)
  const int threads = (list && q.k > kMaxK) ? 128 : 256;
  const size_t walk = size_t(levels) * threads * (STEMS ? 2 * sizeof(A) + 4 : sizeof(A));
  const size_t smem = walk + (list ? size_t(q.k) * threads * (sizeof(A) + sizeof(uint32_t)) : 0);
  return with_dims(t.dims, [&](auto kk) -> cudaError_t {
    constexpr int K = decltype(kk)::value;
    if constexpr (!thread_engine_dims(K)) {
      return cudaErrorInvalidValue;
    } else {
      return with_metric(q.metric, [&](auto m) {
        using M = decltype(m);
        return with_excl(q.exclusive, [&](auto ex) {
          constexpr bool EX = decltype(ex)::value;
          if (!M::kPeriodic && q.periodic) return cudaErrorInvalidValue;
          if constexpr (M::kPeriodic) if (q.periodic) {
            const auto box = make_box<A, K>(q);
            if constexpr (STEMS == 1) {
              if (q.family == KGPU_NEAREST_ONE) {
                // home query plus images, per-thread walks over Donnelly stems
                const size_t nsmem = size_t(levels) * 256 * (2 * sizeof(A) + 4);
                auto kern = k_tperiodic_nn1<A, K, M, STEMS>;
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(nsmem));
                const int grid = grid_for(kern, nsmem, (q.nq + 31) / 32);
                kern<<<grid, 256, nsmem, q.stream>>>(tv, b, box, levels,
                                                     static_cast<A*>(q.out_d), q.out_i, q.out_c,
                                                     q.stats);
                g_launches++;
                return cudaGetLastError();
              }
            }
            if (q.family != KGPU_NEAREST_N && q.family != KGPU_NEAREST_N_WITHIN)
              return cudaErrorInvalidValue;
            // periodic nearest_n: per-thread walk, cooperative leaf scans,
            // lists in the output rows
            const size_t psmem = periodic_smem<A>(t, STEMS);
            auto kern = k_tperiodic_nn<A, K, M, EX, STEMS>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(psmem));
            const int grid = grid_for(kern, psmem, (q.nq + 31) / 32);
            kern<<<grid, 256, psmem, q.stream>>>(tv, b, box, q.k, radius,
                                                  static_cast<A*>(q.out_d), q.out_i, q.out_c,
                                                  q.stats);
            g_launches++;
            return cudaGetLastError();
          }
          auto runt = [&](auto kern) {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            const int grid = grid_for(kern, smem, (q.nq + 31) / 32, threads);
            kern<<<grid, threads, smem, q.stream>>>(tv, b, levels, q.k, radius, q.sorted ? 0 : 1,
                                                static_cast<A*>(q.out_d), q.out_i, q.out_c,
                                                q.stats);
            g_launches++;
            return cudaGetLastError();
          };
          switch (q.family) {
            case KGPU_NEAREST_ONE:
              return runt(k_tfixed<A, K, M, KF_NEAREST_ONE, false, STEMS>);
            case KGPU_APPROX_NEAREST_ONE:  // one straight descent, either stem order
              return runt(k_tfixed<A, K, M, KF_APPROX, false, 0>);
            case KGPU_NEAREST_N:
            case KGPU_NEAREST_N_WITHIN:
              // warp-cooperative leaf scans with lists in the output rows: on
              // request, and by default for f64 lists above 20 entries, where
              // per-thread lists in shared memory cut the blocks per SM (16M
              // queries, f64, k = 24: 95 against 101 ms; k = 32: 115 against
              // 261 ms; f32 up to k = 32 and f64 up to 16 stay per thread)
              if ((q.engine == 3 || (q.engine == 0 && sizeof(A) == 8 && q.k > 20)) && q.sorted &&
                  q.k <= kMaxK) {
                const size_t csmem = size_t(levels) * 256 * (STEMS ? 2 * sizeof(A) + 4 : sizeof(A));
                auto kern = k_tnn_coop<A, K, M, EX, STEMS>;
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(csmem));
                const int grid = grid_for(kern, csmem, (q.nq + 31) / 32);
                kern<<<grid, 256, csmem, q.stream>>>(tv, b, levels, q.k, radius,
                                                     static_cast<A*>(q.out_d), q.out_i, q.out_c,
                                                     q.stats);
                g_launches++;
                return cudaGetLastError();
              }
              return runt(k_tfixed<A, K, M, KF_NEAREST_N, EX, STEMS>);
            case KGPU_BEST_N_WITHIN:
              return runt(k_tfixed<A, K, M, KF_BEST_N, EX, STEMS>);
          }
          return cudaErrorInvalidValue;
        });
      });
    }
  });
}

template <typename A>
cudaError_t launch_tfixed(const DeviceTree& t, const QueryLaunch& q) {
  if (t.scalar_walk()) return launch_tfixed_donnelly(t, q, A());
  return launch_tfixed_stems<A, 0>(t, q);
}

// Lists in the output rows (k_trow, k_tperiodic_row): nearest_n and
// best_n_within of any length on 2-D and 3-D trees, either stem order;
// periodic nearest_n on Eytzinger trees.
template <typename A>
cudaError_t launch_trow(const DeviceTree& t, const QueryLaunch& q) {
  const TreeView<A> tv = make_view<A>(t);
  const Batch<A> b = make_batch<A>(q);
  const A radius = A(q.radius);
  const int levels = t.max_stem_level + 2;
  const bool best = q.family == KGPU_BEST_N_WITHIN;
  return with_dims(t.dims, [&](auto kk) -> cudaError_t {
    constexpr int K = decltype(kk)::value;
    if constexpr (!thread_engine_dims(K)) {
      return cudaErrorInvalidValue;
    } else {
      return with_metric(q.metric, [&](auto m) {
        using M = decltype(m);
        return with_excl(q.exclusive, [&](auto ex) -> cudaError_t {
          constexpr bool EX = decltype(ex)::value;
          if (q.periodic) {
            if constexpr (M::kPeriodic) {
              if (best) return cudaErrorInvalidValue;
              const auto box = make_box<A, K>(q);
              const int stems = t.scalar_walk() ? 1 : 0;
              const size_t smem = periodic_smem<A>(t, stems);
              auto launch = [&](auto kern) {
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(smem));
                const int grid = grid_for(kern, smem, (q.nq + 31) / 32);
                kern<<<grid, 256, smem, q.stream>>>(tv, b, box, q.k, radius,
                                                    static_cast<A*>(q.out_d), q.out_i, q.out_c,
                                                    q.stats);
                g_launches++;
                return cudaGetLastError();
              };
              return stems ? launch(k_tperiodic_row<A, K, M, EX, 1>)
                           : launch(k_tperiodic_row<A, K, M, EX, 0>);
            } else {
              return cudaErrorInvalidValue;
            }
          }
          auto run = [&](auto kern, int stems) {
            const size_t smem =
                size_t(levels) * 256 * (stems ? 2 * sizeof(A) + 4 : sizeof(A));
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            const int grid = grid_for(kern, smem, (q.nq + 31) / 32);
            kern<<<grid, 256, smem, q.stream>>>(tv, b, levels, q.k, best ? 1 : 0, radius,
                                                static_cast<A*>(q.out_d), q.out_i, q.out_c,
                                                q.stats);
            g_launches++;
            return cudaGetLastError();
          };
          if (t.scalar_walk()) return run(k_trow<A, K, M, EX, 1>, 1);
          return run(k_trow<A, K, M, EX, 0>, 0);
        });
      });
    }
  });
}

// Counting (offsets == nullptr, counts set) or filling pass of the radius
// families.
template <typename A, int STEMS>
cudaError_t launch_within_pass_stems(const DeviceTree& t, const QueryLaunch& q, uint64_t* counts,
                                     const uint64_t* offsets) {
  const TreeView<A> tv = make_view<A>(t);
  const Batch<A> b = make_batch<A>(q);
  const A radius = A(q.radius);
  return with_dims(t.dims, [&](auto kk) {
    constexpr int K = decltype(kk)::value;
    return with_metric(q.metric, [&](auto m) {
      using M = decltype(m);
      return with_excl(q.exclusive, [&](auto ex) -> cudaError_t {
        constexpr bool EX = decltype(ex)::value;
        if (!M::kPeriodic && q.periodic) return cudaErrorInvalidValue;
        if constexpr (thread_engine_dims(K) && M::kPeriodic) {
          if (q.periodic && (q.engine != 1 || STEMS)) {
            const auto box = make_box<A, K>(q);
            const size_t smem = periodic_smem<A>(t, STEMS);
            auto kern = k_tperiodic_within<A, K, M, EX, STEMS>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            const int grid = grid_for(kern, smem, (q.nq + 31) / 32);
            kern<<<grid, 256, smem, q.stream>>>(tv, b, box, radius, counts, offsets, q.capacity,
                                                static_cast<A*>(q.out_d), q.out_i, q.status,
                                                q.stats);
            g_launches++;
            return cudaGetLastError();
          }
        }
        if constexpr (M::kPeriodic) if (q.periodic) {
          const auto box = make_box<A, K>(q);
          if (!offsets) {
            auto kern = k_periodic_within_count<A, K, M, EX>;
            kern<<<grid_for(kern, 0, q.nq), 256, 0, q.stream>>>(tv, b, box, radius, counts,
                                                                 q.stats);
          } else {
            auto kern = k_periodic_within_fill<A, K, M, EX>;
            kern<<<grid_for(kern, 0, q.nq), 256, 0, q.stream>>>(
                tv, b, box, radius, offsets, q.capacity, static_cast<A*>(q.out_d), q.out_i,
                q.status);
          }
          g_launches++;
          return cudaGetLastError();
        }
        if constexpr (thread_engine_dims(K)) {
          if (q.engine != 1 || STEMS) {
            const size_t smem = size_t(t.max_stem_level + 2) * 256 *
                                (STEMS ? 2 * sizeof(A) + 4 : sizeof(A));
            auto kern = k_twithin<A, K, M, EX, STEMS>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            const int grid = grid_for(kern, smem, (q.nq + 31) / 32);
            kern<<<grid, 256, smem, q.stream>>>(tv, b, radius, counts, offsets, q.capacity,
                                                static_cast<A*>(q.out_d), q.out_i, q.status,
                                                q.stats);
            g_launches++;
            return cudaGetLastError();
          }
        }
        if (!offsets) {
          auto kern = k_within_count<A, K, M, EX>;
          kern<<<grid_for(kern, 0, q.nq), 256, 0, q.stream>>>(tv, b, radius, counts, q.stats);
        } else {
          auto kern = k_within_fill<A, K, M, EX>;
          kern<<<grid_for(kern, 0, q.nq), 256, 0, q.stream>>>(
              tv, b, radius, offsets, q.capacity, static_cast<A*>(q.out_d), q.out_i, q.status);
        }
        g_launches++;
        return cudaGetLastError();
      });
    });
  });
}

template <typename A>
cudaError_t launch_within_count(const DeviceTree& t, const QueryLaunch& q, uint64_t* counts) {
  if (t.scalar_walk()) return launch_within_donnelly(t, q, counts, nullptr, A());
  return launch_within_pass_stems<A, 0>(t, q, counts, nullptr);
}

template <typename A>
cudaError_t launch_within_fill(const DeviceTree& t, const QueryLaunch& q,
                               const uint64_t* offsets) {
  if (t.scalar_walk()) return launch_within_donnelly(t, q, nullptr, offsets, A());
  return launch_within_pass_stems<A, 0>(t, q, nullptr, offsets);
}

template <typename A>
cudaError_t launch_seg_sort(const uint64_t* offsets, uint64_t nq, uint64_t capacity, A* d,
                            uint32_t* it, A* scratch_d, uint32_t* scratch_i, cudaStream_t s) {
  if (nq == 0) return cudaSuccess;
  {
    auto kern = k_seg_sort_warp<A>;
    const int grid = grid_for(kern, 0, (nq + 31) / 32);
    kern<<<grid, 256, 0, s>>>(offsets, nq, capacity, d, it);
    g_launches++;
  }
  {
    // shared-memory ping-pong buffers for segments up to `cap` hits
    const uint32_t cap = 4096;
    const size_t smem = size_t(cap) * 2 * (sizeof(A) + sizeof(uint32_t));
    auto kern = k_seg_sort_block<A>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    const uint64_t blocks = (nq + 255) / 256;
    kern<<<unsigned(blocks), 256, smem, s>>>(offsets, nq, capacity, d, it, scratch_d, scratch_i,
                                             cap);
    g_launches++;
  }
  return cudaGetLastError();
}

template <typename A>
cudaError_t launch_spatial_order(const DeviceTree& t, const QueryLaunch& q, uint32_t* order,
                                 void* scratch) {
  const TreeView<A> tv = make_view<A>(t);
  const Batch<A> b = make_batch<A>(q);
  const uint64_t nq = q.nq;
  const uint64_t nl = q.forest ? q.total_leaves : (t.leaf_count > 0 ? t.leaf_count : 1);
  // scratch layout: leaf_of[nq] u32 | counts[nl + 1] u64 | scan tiles
  uint8_t* p = static_cast<uint8_t*>(scratch);
  uint32_t* leaf_of = reinterpret_cast<uint32_t*>(p);
  p += ((nq * 4 + 255) / 256) * 256;
  unsigned long long* counts = reinterpret_cast<unsigned long long*>(p);
  p += (((nl + 1) * 8 + 255) / 256) * 256;
  void* tiles = p;
  cudaError_t e = cudaMemsetAsync(counts, 0, (nl + 1) * 8, q.stream);
  if (e != cudaSuccess) return e;
  e = with_dims(t.dims, [&](auto kk) {
    constexpr int K = decltype(kk)::value;
    auto kern = k_leaf_histogram<A, K>;
    const int grid = grid_for(kern, 0, (nq + 31) / 32);
    kern<<<grid, 256, 0, q.stream>>>(tv, b, q.forest ? q.leaf_base : nullptr, leaf_of, counts);
    g_launches++;
    return cudaGetLastError();
  });
  if (e != cudaSuccess) return e;
  e = launch_exclusive_scan(reinterpret_cast<uint64_t*>(counts),
                            reinterpret_cast<uint64_t*>(counts), nl, tiles, q.stream);
  if (e != cudaSuccess) return e;
  {
    auto kern = k_leaf_scatter;
    const int grid = grid_for(kern, 0, (nq + 31) / 32);
    kern<<<grid, 256, 0, q.stream>>>(leaf_of, nq, counts, order);
    g_launches++;
  }
  return cudaGetLastError();
}

}  // namespace kgpu

#define KGPU_INSTANTIATE_WARP(A)                                                                 \
  namespace kgpu {                                                                               \
  template cudaError_t launch_wfixed<A>(const DeviceTree&, const QueryLaunch&);                  \
  }

#define KGPU_INSTANTIATE_THREAD(A)                                                               \
  namespace kgpu {                                                                               \
  template cudaError_t launch_tfixed<A>(const DeviceTree&, const QueryLaunch&);                  \
  }

#define KGPU_INSTANTIATE_DONNELLY(A)                                                             \
  namespace kgpu {                                                                               \
  cudaError_t launch_tfixed_donnelly(const DeviceTree& t, const QueryLaunch& q, A) {             \
    return launch_tfixed_stems<A, 1>(t, q);                                                      \
  }                                                                                              \
  cudaError_t launch_within_donnelly(const DeviceTree& t, const QueryLaunch& q, uint64_t* counts, \
                                     const uint64_t* offsets, A) {                               \
    return launch_within_pass_stems<A, 1>(t, q, counts, offsets);                                \
  }                                                                                              \
  }

#define KGPU_INSTANTIATE_ROWS(A)                                                                 \
  namespace kgpu {                                                                               \
  template cudaError_t launch_trow<A>(const DeviceTree&, const QueryLaunch&);                    \
  }

#define KGPU_INSTANTIATE_RADIUS(A)                                                               \
  namespace kgpu {                                                                               \
  template cudaError_t launch_within_count<A>(const DeviceTree&, const QueryLaunch&, uint64_t*); \
  template cudaError_t launch_within_fill<A>(const DeviceTree&, const QueryLaunch&,              \
                                             const uint64_t*);                                   \
  template cudaError_t launch_seg_sort<A>(const uint64_t*, uint64_t, uint64_t, A*, uint32_t*,    \
                                          A*, uint32_t*, cudaStream_t);                          \
  template cudaError_t launch_spatial_order<A>(const DeviceTree&, const QueryLaunch&, uint32_t*, \
                                               void*);                                           \
  }
