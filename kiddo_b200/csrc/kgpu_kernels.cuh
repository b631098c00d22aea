// kgpu_kernels.cuh — kernels of the query engine.  Instantiated per
// coordinate type and engine in the kernels_*.cu translation units.
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "kgpu_device.cuh"
#include "kgpu_launch.h"
#include "kgpu_thread.cuh"
#include "kgpu_coop.cuh"

namespace kgpu {

__device__ __forceinline__ void add_stats(unsigned long long* stats, const TravStats& st) {
  atomicAdd(stats + 0, (unsigned long long)st.stems);
  atomicAdd(stats + 1, (unsigned long long)st.leaves);
  atomicAdd(stats + 2, (unsigned long long)st.points);
}

enum KernelFamily : int {
  KF_NEAREST_ONE = 0,
  KF_APPROX = 1,
  KF_NEAREST_N = 2,
  KF_BEST_N = 3,
};

// The batch a kernel answers.  Single tree: `tv`; several trees: query qi
// belongs to forest[tree_of[qi]].  radii (if set) gives each query its own
// radius.  With `work` set, warps take queries from that device counter (a
// work queue) instead of a fixed grid stride, which balances batches whose
// queries cost very different amounts.
template <typename A>
struct Batch {
  const A* __restrict__ Q;
  const uint32_t* __restrict__ order;
  uint64_t nq;
  const TreeView<A>* __restrict__ forest;
  const uint32_t* __restrict__ tree_of;
  uint32_t n_trees;
  const A* __restrict__ radii;
  unsigned long long* __restrict__ work;
  // lane-refilled drivers: queries handed to a warp at a time, and idle lanes
  // a warp waits for before it refills them (kgpu_query_desc::tuning)
  uint32_t chunk;
  int refill;
  // when set, a device count that bounds nq (a compacted `order` list whose
  // length the host has not read)
  const unsigned long long* nq_dev = nullptr;

  // the number of queries to process: nq, or less when nq_dev says so
  __device__ __forceinline__ uint64_t count() const {
    if (!nq_dev) return nq;
    const uint64_t m = *nq_dev;
    return m < nq ? m : nq;
  }

  // A query naming no tree of the forest sees an empty tree (no results).
  __device__ __forceinline__ TreeView<A> tree(const TreeView<A>& tv, uint64_t qi) const {
    if (!forest) return tv;
    const uint32_t t = tree_of[qi];
    if (t < n_trees) return forest[t];
    TreeView<A> empty = tv;
    empty.size = 0;
    empty.leaf_count = 0;
    return empty;
  }
  __device__ __forceinline__ A radius(A r, uint64_t qi) const { return radii ? radii[qi] : r; }
  template <int K>
  __device__ __forceinline__ void query(uint64_t qi, A (&q)[K]) const {
#pragma unroll
    for (int d = 0; d < K; ++d) q[d] = __ldg(Q + qi * K + d);
  }
};

// One query per warp: f(qi) with all 32 lanes.
template <typename A, typename F>
__device__ __forceinline__ void for_each_query_warp(const Batch<A>& b, F&& f) {
  const uint64_t nq = b.count();
  if (b.work) {
    const int lane = threadIdx.x & 31;
    for (;;) {
      unsigned long long w = 0;
      if (lane == 0) w = atomicAdd(b.work, 1ull);
      w = __shfl_sync(FULL, w, 0);
      if (w >= nq) break;
      f(b.order ? uint64_t(b.order[w]) : uint64_t(w));
    }
  } else {
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t w = warp; w < nq; w += nwarps) f(b.order ? uint64_t(b.order[w]) : w);
  }
}

// One query per thread; with a work counter a warp takes 32 consecutive slots.
template <typename A, typename F>
__device__ __forceinline__ void for_each_query_thread(const Batch<A>& b, F&& f) {
  const uint64_t nq = b.count();
  if (b.work) {
    const int lane = threadIdx.x & 31;
    for (;;) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(b.work, 32ull);
      base = __shfl_sync(FULL, base, 0);
      if (base >= nq) break;
      const uint64_t w = base + lane;
      if (w < nq) f(b.order ? uint64_t(b.order[w]) : w);
    }
  } else {
    for (uint64_t w = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; w < nq;
         w += uint64_t(gridDim.x) * blockDim.x)
      f(b.order ? uint64_t(b.order[w]) : w);
  }
}

// ---------------------------------------------------------------------------
// Fixed-size families, one warp per query.
// ---------------------------------------------------------------------------
template <typename A, int K, typename M, int FAM, bool EXCL>
__global__ void __launch_bounds__(256) k_fixed(TreeView<A> tv0, Batch<A> b, int k, A radius0,
                                               int arrival_order, A* __restrict__ out_d,
                                               uint32_t* __restrict__ out_i,
                                               uint32_t* __restrict__ out_c,
                                               unsigned long long* __restrict__ stats) {
  const int lane = threadIdx.x & 31;
  for_each_query_warp(b, [&](uint64_t qi) {
    const TreeView<A> tv = b.tree(tv0, qi);
    const A radius = b.radius(radius0, qi);
    A q[K];
    b.query(qi, q);
    TravStats st;
    if constexpr (FAM == KF_NEAREST_ONE) {
      NearestOnePolicy<A, K, M> pol;
      warp_arith_query<A, K, M>(tv, q, pol, lane, st);
      if (lane == 0) {
        out_d[qi] = pol.best;
        out_i[qi] = pol.item;
        if (out_c) out_c[qi] = 1;
      }
    } else if constexpr (FAM == KF_APPROX) {
      A best = inf_of<A>();
      uint32_t item = 0;
      if (tv.leaf_count > 0) {
        st.points = scan_nearest_one<A, K, M>(tv, straight_leaf<A, K>(tv, q), q, lane, best, item);
        st.stems = uint32_t(tv.max_stem_level + 1);
        st.leaves = 1;
      }
      if (lane == 0) {
        out_d[qi] = best;
        out_i[qi] = item;
        if (out_c) out_c[qi] = 1;
      }
    } else if constexpr (FAM == KF_NEAREST_N) {
      NearestNPolicy<A, K, M, EXCL> pol(k, radius);
      warp_arith_query<A, K, M>(tv, q, pol, lane, st);
      pol.write(qi, out_d, out_i, out_c, arrival_order != 0, lane);
    } else {
      BestNPolicy<A, K, M, EXCL> pol(k, radius);
      warp_arith_query<A, K, M>(tv, q, pol, lane, st);
      pol.write(qi, out_d, out_i, out_c, lane);
    }
    if (stats && lane == 0) add_stats(stats, st);
  });
}

// nearest_n and best_n_within with 32 < k <= kMaxBigK, one query per warp,
// each warp's list in its own region of dynamic shared memory: k distances,
// then (after every warp's distances) k items and k arrival numbers per warp.
template <typename A, int K, typename M, int FAM, bool EXCL>
__global__ void __launch_bounds__(256) k_fixed_bign(TreeView<A> tv0, Batch<A> b, int k, A radius0,
                                                    int arrival_order, A* __restrict__ out_d,
                                                    uint32_t* __restrict__ out_i,
                                                    uint32_t* __restrict__ out_c,
                                                    unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char bsmem[];
  const int lane = threadIdx.x & 31;
  const size_t warps = blockDim.x >> 5, w = threadIdx.x >> 5;
  A* ld = reinterpret_cast<A*>(bsmem) + w * k;
  uint32_t* li = reinterpret_cast<uint32_t*>(reinterpret_cast<A*>(bsmem) + warps * k) + w * k;
  uint32_t* ls = li + warps * k;
  for_each_query_warp(b, [&](uint64_t qi) {
    const TreeView<A> tv = b.tree(tv0, qi);
    A q[K];
    b.query(qi, q);
    TravStats st;
    using Pol = typename std::conditional<FAM == KF_BEST_N, BestNBigPolicy<A, K, M, EXCL>,
                                          NearestNBigPolicy<A, K, M, EXCL>>::type;
    Pol pol(ld, li, ls, k, b.radius(radius0, qi));
    warp_arith_query<A, K, M>(tv, q, pol, lane, st);
    pol.write(qi, out_d, out_i, out_c, arrival_order != 0, lane);
    __syncwarp();
    if (stats && lane == 0) add_stats(stats, st);
  });
}

// ---------------------------------------------------------------------------
// Radius families: count pass, exclusive scan, fill pass, segmented sort.
// The fill pass writes at most `cap` hits per query; a query whose count
// differs from its segment (the caller passed offsets of another batch) sets
// *status to KGPU_EOVERFLOW.
// ---------------------------------------------------------------------------
template <typename A, int K, typename M, bool EXCL>
__global__ void __launch_bounds__(256) k_within_count(TreeView<A> tv0, Batch<A> b, A radius0,
                                                      uint64_t* __restrict__ counts,
                                                      unsigned long long* __restrict__ stats) {
  const int lane = threadIdx.x & 31;
  for_each_query_warp(b, [&](uint64_t qi) {
    const TreeView<A> tv = b.tree(tv0, qi);
    A q[K];
    b.query(qi, q);
    WithinCountPolicy<A, K, M, EXCL> pol(b.radius(radius0, qi));
    TravStats st;
    warp_arith_query<A, K, M>(tv, q, pol, lane, st);
    if (lane == 0) counts[qi] = pol.count;
    if (stats && lane == 0) add_stats(stats, st);
  });
}

template <typename A, int K, typename M, bool EXCL>
__global__ void __launch_bounds__(256) k_within_fill(TreeView<A> tv0, Batch<A> b, A radius0,
                                                     const uint64_t* __restrict__ offsets,
                                                     uint64_t capacity, A* __restrict__ out_d,
                                                     uint32_t* __restrict__ out_i,
                                                     int* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  for_each_query_warp(b, [&](uint64_t qi) {
    const uint64_t o = offsets[qi];
    const uint64_t end = offsets[qi + 1] < capacity ? offsets[qi + 1] : capacity;
    if (end <= o) return;
    const TreeView<A> tv = b.tree(tv0, qi);
    A q[K];
    b.query(qi, q);
    WithinFillPolicy<A, K, M, EXCL> pol(b.radius(radius0, qi), end - o, out_d + o, out_i + o);
    TravStats st;
    warp_arith_query<A, K, M>(tv, q, pol, lane, st);
    if (lane == 0 && status && pol.count != offsets[qi + 1] - o) atomicExch(status, 6);
  });
}

// ---------------------------------------------------------------------------
// Thread-per-query kernels.  Dynamic shared memory: one continuation slot per
// level per thread, (max_stem_level + 2) * blockDim values of A.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void flush_stats(unsigned long long* stats, const TravStats& st) {
  const unsigned s0 = __reduce_add_sync(FULL, st.stems);
  const unsigned s1 = __reduce_add_sync(FULL, st.leaves);
  const unsigned s2 = __reduce_add_sync(FULL, st.points);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(stats + 0, (unsigned long long)s0);
    atomicAdd(stats + 1, (unsigned long long)s1);
    atomicAdd(stats + 2, (unsigned long long)s2);
  }
}

// Queries handed out to the lanes of one warp in chunks of Batch::chunk
// queries (64 unless tuned): from the batch's work counter when it has one,
// else chunks gw, gw + W, gw + 2W, ... (gw = this warp, W = warps in the
// grid).  Interleaving spreads the costly regions of a leaf-ordered batch
// evenly over the warps.
struct LaneFeeder {
  uint64_t next, end, chunk, step;
  bool done;

  __device__ __forceinline__ void start() {
    step = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    chunk = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    next = end = 0;
    done = false;
  }

  // Warp-uniform: moves to the next chunk; false once the batch is used up.
  template <typename A>
  __device__ __forceinline__ bool advance(const Batch<A>& b) {
    if (done) return false;
    uint64_t base;
    const uint64_t n = b.chunk;
    if (b.work) {
      unsigned long long v = 0;
      if ((threadIdx.x & 31) == 0) v = atomicAdd(b.work, (unsigned long long)n);
      base = __shfl_sync(FULL, v, 0);
    } else {
      base = chunk * n;
      chunk += step;
    }
    const uint64_t nq = b.count();
    if (base >= nq) {
      done = true;
      return false;
    }
    next = base;
    end = base + n < nq ? base + n : nq;
    return true;
  }
};

// Warp-uniform: once at least Batch::refill lanes of the warp (24 unless
// tuned), or all of them, have no query, gives each of them the next query of
// the batch (lowest lanes first, so new queries start side by side); returns
// whether any lane of the warp still has a query.
template <typename A>
__device__ __forceinline__ bool refill_lanes(const Batch<A>& b, LaneFeeder& fd, bool& active,
                                             bool& fresh, uint64_t& qi) {
  const unsigned lane = threadIdx.x & 31;
  unsigned need = __ballot_sync(FULL, !active);
  if (need != FULL && __popc(need) < b.refill) return true;
  while (need) {
    if (fd.next >= fd.end && !fd.advance(b)) break;
    const uint64_t avail = fd.end - fd.next;
    const int cnt = __popc(need);
    const int take = avail < uint64_t(cnt) ? int(avail) : cnt;
    if (!active) {
      const int rank = __popc(need & ((1u << lane) - 1u));
      if (rank < take) {
        const uint64_t w = fd.next + uint64_t(rank);
        qi = b.order ? uint64_t(b.order[w]) : w;
        active = fresh = true;
      }
    }
    fd.next += uint64_t(take);
    need = __ballot_sync(FULL, !active);
  }
  return __any_sync(FULL, active);
}

// ---------------------------------------------------------------------------
// The driver: lane-refilled per-thread walks, cooperative leaf scans.
//   start(qi, tv) sets the policy up for a fresh query in this lane and says
//   whether the query needs a walk at all; finish(o, qi) runs on the whole
//   warp for lane o's finished query.
// ---------------------------------------------------------------------------
template <typename A, int K, typename M, typename Walk, typename Pol, typename Start,
          typename Finish>
__device__ __forceinline__ void coop_drive(const TreeView<A>& tv0, const Batch<A>& b, Walk& wk,
                                           Pol& pol, A* __restrict__ slot, int stride,
                                           TravStats& st, Start&& start, Finish&& finish) {
  const int lane = threadIdx.x & 31;
  LaneFeeder fd;
  fd.start();
  TreeView<A> tv = tv0;
  A q[K];
#pragma unroll
  for (int d = 0; d < K; ++d) q[d] = A(0);
  bool active = false, fresh = false;
  uint64_t qi = 0;
  for (;;) {
    bool done = false;
    if (active && !wk.backtrack(tv, q, pol, slot, stride)) {
      done = true;
      active = false;
    }
    for (unsigned fm = __ballot_sync(FULL, done); fm; fm &= fm - 1) {
      const int o = __ffs(fm) - 1;
      finish(o, shfl64(qi, o));
    }
    if (!refill_lanes(b, fd, active, fresh, qi)) break;
    bool bounded = true, empty = false;
    if (fresh) {
      fresh = false;
      tv = b.tree(tv0, qi);
      b.query(qi, q);
      wk.init();
      if (!start(qi, tv)) {
        active = false;
      } else if (tv.size == 0) {
        empty = true;
        active = false;
      }
      bounded = !pol.unbounded_start();
    }
    for (unsigned fm = __ballot_sync(FULL, empty); fm; fm &= fm - 1) {
      const int o = __ffs(fm) - 1;
      finish(o, shfl64(qi, o));
    }
    const uint8_t* lb = nullptr;
    uint32_t len = 0;
    if (active) {
      const uint32_t leaf = wk.descend(tv, q, pol, bounded, slot, stride, st);
      const uint2 ex = wk.leaf_extents(tv, leaf);
      lb = tv.arena + size_t(ex.x) * 8;
      len = ex.y;
      st.points += len;
      ++st.leaves;
    }
    for (unsigned lm = __ballot_sync(FULL, active); lm; lm &= lm - 1) {
      const int o = __ffs(lm) - 1;
      pol.leaf(o, shfl64(qi, o), coop_leaf<A, K>(o, lb, len, q), lane);
    }
  }
}


// The per-thread driver: lane-refilled walks, each thread scanning its own
// leaves (the list families keep their lists in shared-memory columns).
//   finish(qi) writes a finished query's results from its own lane.
template <typename A, int K, typename M, bool kForest, typename Walk, typename Pol,
          typename Finish>
__device__ __forceinline__ void thread_drive_impl(const TreeView<A>& tv0, const Batch<A>& b,
                                                  A radius0, Walk& wk, Pol& pol,
                                                  A* __restrict__ slot, int stride, TravStats& st,
                                                  Finish&& finish) {
  LaneFeeder fd;
  fd.start();
  TreeView<A> tv = tv0;
  A q[K];
#pragma unroll
  for (int d = 0; d < K; ++d) q[d] = A(0);
  bool active = false, fresh = false;
  uint64_t qi = 0;
  for (;;) {
    if (active && !wk.backtrack(tv, q, pol, slot, stride)) {
      finish(qi);
      active = false;
    }
    if (!refill_lanes(b, fd, active, fresh, qi)) break;
    bool bounded = true;
    if (fresh) {
      fresh = false;
      if constexpr (kForest) tv = b.tree(tv0, qi);
      b.query(qi, q);
      pol.reset(b.radius(radius0, qi));
      wk.init();
      bounded = !pol.unbounded_start();
      if (tv.size == 0) {
        finish(qi);
        active = false;
      }
    }
    if (active) {
      const uint32_t leaf = wk.descend(tv, q, pol, bounded, slot, stride, st);
      st.points += pol.leaf(tv, wk.leaf_extents(tv, leaf), q);
      ++st.leaves;
    }
  }
}

// One copy of the driver for a batch over one tree, where every lane's tree
// is the kernel's own argument (no per-lane tree state held in registers), and
// one for a forest batch, where each query names its tree.  (The cooperative
// driver keeps one copy: with two, the 256-catalogue forest's radius queries
// ran 8% slower.)
template <typename A, int K, typename M, typename Walk, typename Pol, typename Finish>
__device__ __forceinline__ void thread_drive(const TreeView<A>& tv0, const Batch<A>& b, A radius0,
                                             Walk& wk, Pol& pol, A* __restrict__ slot, int stride,
                                             TravStats& st, Finish&& finish) {
  if (b.forest)
    thread_drive_impl<A, K, M, true>(tv0, b, radius0, wk, pol, slot, stride, st, finish);
  else
    thread_drive_impl<A, K, M, false>(tv0, b, radius0, wk, pol, slot, stride, st, finish);
}

// The per-thread walk of a stem order: Eytzinger arithmetic DFS (STEMS == 0)
// or Donnelly scalar backtracking (STEMS == 1).  Shared memory begins with the
// walk's per-level columns: rd slots for both, then for Donnelly the off
// values and the far stem indices.
template <typename A, int K, typename M, int STEMS>
struct WalkOf {
  using type = ThreadWalk<A, K, M>;
  __device__ static type make(unsigned char*, int, int) { return type(); }
  __host__ __device__ static size_t bytes(int levels, int stride) {
    return size_t(levels) * stride * sizeof(A);
  }
};
template <typename A, int K, typename M>
struct WalkOf<A, K, M, 1> {
  using type = DonnellyWalk<A, K, M>;
  __device__ static type make(unsigned char* smem, int levels, int stride) {
    A* offs = reinterpret_cast<A*>(smem) + size_t(levels) * stride + threadIdx.x;
    uint32_t* stems = reinterpret_cast<uint32_t*>(reinterpret_cast<A*>(smem) +
                                                  2 * size_t(levels) * stride) + threadIdx.x;
    return type(offs, stems);
  }
  __host__ __device__ static size_t bytes(int levels, int stride) {
    return size_t(levels) * stride * (2 * sizeof(A) + sizeof(uint32_t));
  }
};

#ifndef KGPU_BESTN_COOP
#define KGPU_BESTN_COOP 1
#endif

// Shared memory: the continuation slots ((max_stem_level + 2) * blockDim
// values of A, slot of level L for thread t at L * blockDim + t), then for the
// list families k distances and k items per thread.
//
// The exact families walk one query per thread with lane refill: a lane whose
// query has finished takes the next one once enough lanes of its warp are
// idle, so lanes do not wait for the warp's slowest query.  nearest_one and
// nearest_n scan their leaves per thread; best_n_within scans them
// warp-cooperatively (kgpu_coop.cuh).  Each query's own traversal is unchanged.
// Four 256-thread blocks per SM (64 registers) in general; three (80
// registers, no spills) for best_n and for the f64 nearest_one / nearest_n
// kernels, whose two 16-byte row loads per point would spill at 64.
#ifndef KGPU_TFIXED_MIN_BLOCKS
#define KGPU_TFIXED_MIN_BLOCKS 4
#endif
template <int FAM, typename A>
constexpr int tfixed_min_blocks() {
  return (FAM == KF_BEST_N || ((FAM == KF_NEAREST_N || FAM == KF_NEAREST_ONE) && sizeof(A) == 8))
             ? 3
             : KGPU_TFIXED_MIN_BLOCKS;
}
template <typename A, int K, typename M, int FAM, bool EXCL, int STEMS = 0>
__global__ void __launch_bounds__(256, tfixed_min_blocks<FAM, A>())
    k_tfixed(TreeView<A> tv0, Batch<A> b, int levels, int k, A radius0, int arrival_order,
             A* __restrict__ out_d, uint32_t* __restrict__ out_i, uint32_t* __restrict__ out_c,
             unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char tsmem[];
  const int stride = blockDim.x;
  A* slot = reinterpret_cast<A*>(tsmem) + threadIdx.x;
  using W = WalkOf<A, K, M, STEMS>;
  auto wk = W::make(tsmem, levels, stride);
  // the list families' shared memory follows the walk's columns
  unsigned char* lists = tsmem + W::bytes(levels, stride);
  TravStats st;
  if constexpr (FAM == KF_APPROX) {
    for_each_query_thread(b, [&](uint64_t qi) {
      const TreeView<A> tv = b.tree(tv0, qi);
      A q[K];
      b.query(qi, q);
      TNearestOne<A, K, M> pol;
      if (tv.leaf_count > 0) {
        st.points += pol.leaf(tv, __ldg(tv.extents + straight_leaf<A, K>(tv, q)), q);
        st.stems += uint32_t(tv.max_stem_level + 1);
        st.leaves += 1;
      }
      out_d[qi] = pol.best;
      out_i[qi] = pol.item;
      if (out_c) out_c[qi] = 1;
    });
  } else if constexpr (FAM == KF_NEAREST_ONE) {
    TNearestOne<A, K, M> pol;
    thread_drive<A, K, M>(tv0, b, radius0, wk, pol, slot, stride, st, [&](uint64_t qi) {
      out_d[qi] = pol.best;
      out_i[qi] = pol.item;
      if (out_c) out_c[qi] = 1;
    });
  } else if constexpr (FAM == KF_NEAREST_N || !KGPU_BESTN_COOP) {
    // lists in shared-memory columns: entry j of thread t at j * blockDim + t
    if constexpr (FAM == KF_NEAREST_N) {
      TNearestN<A, K, M, EXCL> pol(lists, stride, k, radius0);
      thread_drive<A, K, M>(tv0, b, radius0, wk, pol, slot, stride, st, [&](uint64_t qi) {
        pol.write(qi, out_d, out_i, out_c, arrival_order != 0);
      });
    } else {
      A* list_d = reinterpret_cast<A*>(lists) + threadIdx.x;
      uint32_t* list_i =
          reinterpret_cast<uint32_t*>(reinterpret_cast<A*>(lists) + size_t(k) * stride) +
          threadIdx.x;
      TBestN<A, K, M, EXCL> pol(list_d, list_i, stride, k, radius0);
      thread_drive<A, K, M>(tv0, b, radius0, wk, pol, slot, stride, st,
                            [&](uint64_t qi) { pol.write(qi, out_d, out_i, out_c); });
    }
  } else {
    // best_n_within with warp-cooperative leaf scans: thread t's k entries
    // consecutive at t * k
    const size_t warp0 = threadIdx.x & ~31u;
    A* lists_d = reinterpret_cast<A*>(lists);
    uint32_t* lists_i = reinterpret_cast<uint32_t*>(lists_d + size_t(k) * stride);
    CBestN<A, K, M, EXCL> pol(lists_d + warp0 * k, lists_i + warp0 * k, nullptr, k, radius0);
    coop_drive<A, K, M>(
        tv0, b, wk, pol, slot, stride, st,
        [&](uint64_t qi, const TreeView<A>&) {
          pol.reset(b.radius(radius0, qi));
          return true;
        },
        [&](int o, uint64_t qo) { pol.finish(o, qo, threadIdx.x & 31, out_d, out_i, out_c); });
  }
  if (stats) flush_stats(stats, st);
}

// nearest_n / nearest_n().within with sorted output, k <= 32: per-thread
// walks with lane refill (coop_drive), every leaf scanned by the whole warp
// for its owner (lane p on point p: one coalesced load of the leaf's rows),
// the owner's list kept sorted in its own output row (CNearestNRow: inserts
// by ballot and shuffle, or a bitonic merge of a chunk's candidates).  Same
// list as the per-thread scan: the k smallest by (distance, arrival).
// Shared memory: the walk's per-level columns only.
#ifndef KGPU_TNN_COOP_MIN_BLOCKS
#define KGPU_TNN_COOP_MIN_BLOCKS 4
#endif
template <typename A, int K, typename M, bool EXCL, int STEMS = 0>
__global__ void __launch_bounds__(256, KGPU_TNN_COOP_MIN_BLOCKS)
    k_tnn_coop(TreeView<A> tv0, Batch<A> b, int levels, int k, A radius0,
               A* __restrict__ out_d, uint32_t* __restrict__ out_i, uint32_t* __restrict__ out_c,
               unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char tsmem[];
  const int stride = blockDim.x;
  const int lane = threadIdx.x & 31;
  A* slot = reinterpret_cast<A*>(tsmem) + threadIdx.x;
  auto wk = WalkOf<A, K, M, STEMS>::make(tsmem, levels, stride);
  TravStats st;
  CNearestNRow<A, K, M, EXCL, CartesianDist<A, K, M>> pol(out_d, out_i, k,
                                                          CartesianDist<A, K, M>());
  coop_drive<A, K, M>(
      tv0, b, wk, pol, slot, stride, st,
      [&](uint64_t qi, const TreeView<A>&) {
        pol.reset(b.radius(radius0, qi));
        return true;
      },
      [&](int o, uint64_t qo) { pol.finish(o, qo, lane, out_c); });
  if (stats) flush_stats(stats, st);
}

// nearest_n (sorted rows) and best_n_within with lists of any length held in
// the output rows (CRowList): per-thread walks over Eytzinger (STEMS == 0) or
// Donnelly (STEMS == 1) stems with lane refill, each leaf scanned by the whole
// warp for its owner.  The path for lists beyond the shared-memory kernels'
// range and for Donnelly trees above 32 entries.  Shared memory: the walk's
// per-level columns only.
template <typename A, int K, typename M, bool EXCL, int STEMS = 0>
__global__ void __launch_bounds__(256) k_trow(TreeView<A> tv0, Batch<A> b, int levels, int k,
                                              int best_n, A radius0, A* __restrict__ out_d,
                                              uint32_t* __restrict__ out_i,
                                              uint32_t* __restrict__ out_c,
                                              unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char tsmem[];
  const int stride = blockDim.x;
  const int lane = threadIdx.x & 31;
  A* slot = reinterpret_cast<A*>(tsmem) + threadIdx.x;
  auto wk = WalkOf<A, K, M, STEMS>::make(tsmem, levels, stride);
  TravStats st;
  CRowList<A, K, M, EXCL, CartesianDist<A, K, M>> pol(best_n != 0, out_d, out_i, k,
                                                      CartesianDist<A, K, M>());
  coop_drive<A, K, M>(
      tv0, b, wk, pol, slot, stride, st,
      [&](uint64_t qi, const TreeView<A>&) {
        pol.reset(b.radius(radius0, qi));
        return true;
      },
      [&](int o, uint64_t qo) { pol.finish(o, qo, lane, out_c); });
  if (stats) flush_stats(stats, st);
}

// Counting pass (offsets == nullptr) or filling pass of the radius families.
template <typename A, int K, typename M, bool EXCL, int STEMS = 0>
__global__ void __launch_bounds__(256) k_twithin(TreeView<A> tv0, Batch<A> b, A radius0,
                                                 uint64_t* __restrict__ counts,
                                                 const uint64_t* __restrict__ offsets,
                                                 uint64_t capacity, A* __restrict__ out_d,
                                                 uint32_t* __restrict__ out_i,
                                                 int* __restrict__ status,
                                                 unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char tsmem[];
  A* slot = reinterpret_cast<A*>(tsmem) + threadIdx.x;
  const int stride = blockDim.x;
  const int lane = threadIdx.x & 31;
  TravStats st;
  CWithin<A, K, M, EXCL> pol;
  // the launch sizes shared memory for max_stem_level + 2 levels
  auto wk = WalkOf<A, K, M, STEMS>::make(tsmem, tv0.max_stem_level + 2, stride);
  uint64_t o = 0;  // this lane's segment start (filling pass)
  coop_drive<A, K, M>(
      tv0, b, wk, pol, slot, stride, st,
      [&](uint64_t qi, const TreeView<A>&) {
        pol.radius = b.radius(radius0, qi);
        pol.count = 0;
        pol.cap = 0;
        pol.out_d = nullptr;
        pol.out_i = nullptr;
        if (!offsets) return true;
        o = offsets[qi];
        const uint64_t end = offsets[qi + 1] < capacity ? offsets[qi + 1] : capacity;
        if (end <= o) return false;  // no hits to place (empty segment, or past the capacity)
        pol.cap = end - o;
        pol.out_d = out_d + o;
        pol.out_i = out_i + o;
        return true;
      },
      [&](int w, uint64_t qo) {
        const uint64_t cnt = shfl64(pol.count, w);
        const uint64_t ow = shfl64(o, w);
        if (lane == 0) {
          if (counts) counts[qo] = cnt;
          if (offsets && status && cnt != offsets[qo + 1] - ow) atomicExch(status, 6);
        }
      });
  if (stats) flush_stats(stats, st);
}

// ---------------------------------------------------------------------------
// Periodic families (kd_tree/query/periodic.rs), one warp per query.
// ---------------------------------------------------------------------------
template <typename A, int K>
struct BoxArg {
  A v[K];
};

// Periodic families, one query per thread: PeriodicWalk with lane refill,
// leaves scanned warp-cooperatively.  Each iteration: finish the lanes whose
// walks ended, refill, take every active walk to its next leaf, scan those.
// Shared memory: the rd slot column ((max_stem_level + 2) * blockDim values
// of A); Donnelly stems (STEMS == 1) add one u32 column of path stem indices
// after it (periodic_smem).
template <typename A, int K, typename M, int STEMS, bool kForest, typename Pol, typename Start,
          typename Finish>
__device__ __forceinline__ void periodic_drive_impl(const TreeView<A>& tv0, const Batch<A>& b,
                                                    const A (&box)[K], Pol& pol,
                                                    A* __restrict__ slot, int stride,
                                                    TravStats& st, Start&& start,
                                                    Finish&& finish) {
  const int lane = threadIdx.x & 31;
  // after the rd slots: for Donnelly stems the path column, then the walk's
  // 3K cell-state columns (periodic_smem)
  extern __shared__ __align__(16) unsigned char psmem[];
  size_t o = size_t(tv0.max_stem_level + 2) * stride * sizeof(A);
  uint32_t* path = nullptr;
  if constexpr (STEMS) {
    path = reinterpret_cast<uint32_t*>(psmem + o) + threadIdx.x;
    o += size_t(tv0.max_stem_level + 2) * stride * sizeof(uint32_t);
  }
  PeriodicWalk<A, K, M, STEMS> wk(path, reinterpret_cast<A*>(psmem + o) + threadIdx.x, stride);
  wk.init(box);
  LaneFeeder fd;
  fd.start();
  TreeView<A> tv = tv0;
  A q[K];
#pragma unroll
  for (int d = 0; d < K; ++d) q[d] = A(0);
  bool active = false, fresh = false, done = false;
  uint64_t qi = 0;
  for (;;) {
    for (unsigned fm = __ballot_sync(FULL, done); fm; fm &= fm - 1) {
      const int o = __ffs(fm) - 1;
      finish(o, shfl64(qi, o));
    }
    done = false;
    if (!refill_lanes(b, fd, active, fresh, qi)) break;
    if (fresh) {
      fresh = false;
      if constexpr (kForest) tv = b.tree(tv0, qi);
      b.query(qi, q);
      wk.init(box);
      if (!start(qi)) {
        active = false;
      } else if (tv.size == 0) {
        done = true;
        active = false;
      }
    }
    const uint8_t* lb = nullptr;
    uint32_t len = 0;
    if (active) {
      const uint32_t leaf = wk.next(tv, q, box, pol, slot, stride, st);
      if (leaf == PeriodicWalk<A, K, M, STEMS>::kDone) {
        done = true;
        active = false;
      } else {
        const uint2 ex = __ldg(tv.extents + leaf);
        lb = tv.arena + size_t(ex.x) * 8;
        len = ex.y;
        st.points += len;
        ++st.leaves;
      }
    }
    for (unsigned lm = __ballot_sync(FULL, active); lm; lm &= lm - 1) {
      const int o = __ffs(lm) - 1;
      pol.leaf(o, shfl64(qi, o), coop_leaf<A, K>(o, lb, len, q), lane);
    }
  }
}

template <typename A, int K, typename M, int STEMS, typename Pol, typename Start,
          typename Finish>
__device__ __forceinline__ void periodic_drive(const TreeView<A>& tv0, const Batch<A>& b,
                                               const A (&box)[K], Pol& pol, A* __restrict__ slot,
                                               int stride, TravStats& st, Start&& start,
                                               Finish&& finish) {
  if (b.forest)
    periodic_drive_impl<A, K, M, STEMS, true>(tv0, b, box, pol, slot, stride, st, start, finish);
  else
    periodic_drive_impl<A, K, M, STEMS, false>(tv0, b, box, pol, slot, stride, st, start, finish);
}

// Periodic nearest_n / nearest_n().within (always sorted, periodic.rs
// into_sorted): shared memory holds one rd slot per level per thread.
#ifndef KGPU_TPERIODIC_MIN_BLOCKS
#define KGPU_TPERIODIC_MIN_BLOCKS 3
#endif
template <typename A, int K, typename M, bool EXCL, int STEMS = 0>
__global__ void __launch_bounds__(256, KGPU_TPERIODIC_MIN_BLOCKS) k_tperiodic_nn(TreeView<A> tv0, Batch<A> b,
                                                      BoxArg<A, K> box, int k, A radius0,
                                                      A* __restrict__ out_d,
                                                      uint32_t* __restrict__ out_i,
                                                      uint32_t* __restrict__ out_c,
                                                      unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char tsmem[];
  A* slot = reinterpret_cast<A*>(tsmem) + threadIdx.x;
  const int lane = threadIdx.x & 31;
  TravStats st;
  PeriodicDist<A, K, M> pd;
#pragma unroll
  for (int d = 0; d < K; ++d) pd.box[d] = box.v[d];
  CNearestNRow<A, K, M, EXCL, PeriodicDist<A, K, M>> pol(out_d, out_i, k, pd);
  periodic_drive<A, K, M, STEMS>(
      tv0, b, box.v, pol, slot, blockDim.x, st,
      [&](uint64_t qi) {
        pol.reset(b.radius(radius0, qi));
        return true;
      },
      [&](int o, uint64_t qo) { pol.finish(o, qo, lane, out_c); });
  if (stats) flush_stats(stats, st);
}

// Periodic nearest_one with per-thread walks (periodic.rs:156-214): the home
// query, then each shifted image whose lower bound beats the home result, in
// stable lower-bound order, skipping those that no longer beat the best so
// far.  Image j of the 3^K shifts has shift digit (j / 3^(K-1-a)) % 3 - 1 on
// axis a, the generation order of periodic_image_candidates (:45-142).  The
// path for Donnelly stems (the warp engine's home and image queries walk
// Eytzinger stems).  Shared memory: the walk's per-level columns.
template <typename A, int K, typename M, int STEMS>
__global__ void __launch_bounds__(256) k_tperiodic_nn1(TreeView<A> tv0, Batch<A> b,
                                                       BoxArg<A, K> box, int levels,
                                                       A* __restrict__ out_d,
                                                       uint32_t* __restrict__ out_i,
                                                       uint32_t* __restrict__ out_c,
                                                       unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char tsmem[];
  const int stride = blockDim.x;
  A* slot = reinterpret_cast<A*>(tsmem) + threadIdx.x;
  auto wk = WalkOf<A, K, M, STEMS>::make(tsmem, levels, stride);
  TravStats st;
  for_each_query_thread(b, [&](uint64_t qi) {
    const TreeView<A> tv = b.tree(tv0, qi);
    A q[K];
    b.query(qi, q);
    // one full nearest_one traversal (the reference's scalar/arithmetic walk)
    auto nearest = [&](const A (&qq)[K], A& best, uint32_t& item) {
      TNearestOne<A, K, M> pol;
      if (tv.size != 0) {
        wk.init();
        uint32_t leaf = wk.descend(tv, qq, pol, !pol.unbounded_start(), slot, stride, st);
        st.points += pol.leaf(tv, wk.leaf_extents(tv, leaf), qq);
        ++st.leaves;
        while (wk.backtrack(tv, qq, pol, slot, stride)) {
          leaf = wk.descend(tv, qq, pol, true, slot, stride, st);
          st.points += pol.leaf(tv, wk.leaf_extents(tv, leaf), qq);
          ++st.leaves;
        }
      }
      best = pol.best;
      item = pol.item;
    };
    A best;
    uint32_t item;
    nearest(q, best, item);
    constexpr int NI = pow3(K);
    A lb[NI];
    uint32_t valid = 0;  // bit j: image j is a candidate (nonzero shift, lb < home best)
#pragma unroll
    for (int j = 0; j < NI; ++j) {
      bool nonzero = false;
      A acc = A(0);
#pragma unroll
      for (int a = 0; a < K; ++a) {
        int div = 1;
        for (int c = a + 1; c < K; ++c) div *= 3;
        const int digit = (j / div) % 3;
        const A L = box.v[a];
        const A w = digit == 0 ? sub_rn(q[a], L) : (digit == 1 ? q[a] : add_rn(q[a], L));
        nonzero |= digit != 1;
        // periodic_image_axis_offset (periodic.rs:29-37)
        const A o = w < A(0) ? abs_val(sub_rn(w, A(0))) : (w > L ? abs_val(sub_rn(w, L)) : A(0));
        acc = M::combine(acc, M::template dist1<A>(o, A(0)));
      }
      lb[j] = acc;
      if (nonzero && acc < best) valid |= 1u << j;
    }
    while (valid) {
      // the next candidate in stable lower-bound order
      int pick = -1;
      for (int j = 0; j < NI; ++j)
        if ((valid >> j) & 1u)
          if (pick < 0 || lb[j] < lb[pick]) pick = j;
      valid &= ~(1u << pick);
      if (!(lb[pick] < best)) continue;
      A img[K];
#pragma unroll
      for (int a = 0; a < K; ++a) {
        int div = 1;
        for (int c = a + 1; c < K; ++c) div *= 3;
        const int digit = (pick / div) % 3;
        const A L = box.v[a];
        img[a] = digit == 0 ? sub_rn(q[a], L) : (digit == 1 ? q[a] : add_rn(q[a], L));
      }
      A d;
      uint32_t it;
      nearest(img, d, it);
      if (d < best) {
        best = d;
        item = it;
      }
    }
    out_d[qi] = best;
    out_i[qi] = item;
    if (out_c) out_c[qi] = 1;
  });
  if (stats) flush_stats(stats, st);
}

// Periodic nearest_n lists of any length in the output rows (CRowList with the
// minimum-image distance); sorted rows, periodic.rs into_sorted_vec.
template <typename A, int K, typename M, bool EXCL, int STEMS = 0>
__global__ void __launch_bounds__(256) k_tperiodic_row(TreeView<A> tv0, Batch<A> b,
                                                       BoxArg<A, K> box, int k, A radius0,
                                                       A* __restrict__ out_d,
                                                       uint32_t* __restrict__ out_i,
                                                       uint32_t* __restrict__ out_c,
                                                       unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char tsmem[];
  A* slot = reinterpret_cast<A*>(tsmem) + threadIdx.x;
  const int lane = threadIdx.x & 31;
  TravStats st;
  PeriodicDist<A, K, M> pd;
#pragma unroll
  for (int d = 0; d < K; ++d) pd.box[d] = box.v[d];
  CRowList<A, K, M, EXCL, PeriodicDist<A, K, M>> pol(false, out_d, out_i, k, pd);
  periodic_drive<A, K, M, STEMS>(
      tv0, b, box.v, pol, slot, blockDim.x, st,
      [&](uint64_t qi) {
        pol.reset(b.radius(radius0, qi));
        return true;
      },
      [&](int o, uint64_t qo) { pol.finish(o, qo, lane, out_c); });
  if (stats) flush_stats(stats, st);
}

// Periodic within: counting pass (offsets == nullptr) or filling pass.
template <typename A, int K, typename M, bool EXCL, int STEMS = 0>
__global__ void __launch_bounds__(256, KGPU_TPERIODIC_MIN_BLOCKS) k_tperiodic_within(
    TreeView<A> tv0, Batch<A> b, BoxArg<A, K> box, A radius0, uint64_t* __restrict__ counts,
    const uint64_t* __restrict__ offsets, uint64_t capacity, A* __restrict__ out_d,
    uint32_t* __restrict__ out_i, int* __restrict__ status,
    unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char tsmem[];
  A* slot = reinterpret_cast<A*>(tsmem) + threadIdx.x;
  const int lane = threadIdx.x & 31;
  TravStats st;
  PeriodicDist<A, K, M> pd;
#pragma unroll
  for (int d = 0; d < K; ++d) pd.box[d] = box.v[d];
  CWithin<A, K, M, EXCL, PeriodicDist<A, K, M>> pol(pd);
  uint64_t o = 0;  // this lane's segment start (filling pass)
  periodic_drive<A, K, M, STEMS>(
      tv0, b, box.v, pol, slot, blockDim.x, st,
      [&](uint64_t qi) {
        pol.radius = b.radius(radius0, qi);
        pol.count = 0;
        pol.cap = 0;
        pol.out_d = nullptr;
        pol.out_i = nullptr;
        if (!offsets) return true;
        o = offsets[qi];
        const uint64_t end = offsets[qi + 1] < capacity ? offsets[qi + 1] : capacity;
        if (end <= o) return false;  // no hits to place (empty segment, or past the capacity)
        pol.cap = end - o;
        pol.out_d = out_d + o;
        pol.out_i = out_i + o;
        return true;
      },
      [&](int w, uint64_t qo) {
        const uint64_t cnt = shfl64(pol.count, w);
        const uint64_t ow = shfl64(o, w);
        if (lane == 0) {
          if (counts) counts[qo] = cnt;
          if (offsets && status && cnt != offsets[qo + 1] - ow) atomicExch(status, 6);
        }
      });
  if (stats) flush_stats(stats, st);
}

template <typename A, int K, typename M, int FAM, bool EXCL>
__global__ void __launch_bounds__(256) k_periodic_fixed(TreeView<A> tv0, Batch<A> b,
                                                        BoxArg<A, K> box, int k, A radius0,
                                                        A* __restrict__ out_d,
                                                        uint32_t* __restrict__ out_i,
                                                        uint32_t* __restrict__ out_c,
                                                        unsigned long long* __restrict__ stats) {
  const int lane = threadIdx.x & 31;
  for_each_query_warp(b, [&](uint64_t qi) {
    const TreeView<A> tv = b.tree(tv0, qi);
    A q[K];
    b.query(qi, q);
    TravStats st;
    if constexpr (FAM == KF_NEAREST_ONE) {
      A best;
      uint32_t item;
      warp_periodic_nearest_one<A, K, M>(tv, q, box.v, lane, best, item, st);
      if (lane == 0) {
        out_d[qi] = best;
        out_i[qi] = item;
        if (out_c) out_c[qi] = 1;
      }
    } else {
      PeriodicDist<A, K, M> pd;
#pragma unroll
      for (int d = 0; d < K; ++d) pd.box[d] = box.v[d];
      NearestNPolicy<A, K, M, EXCL, PeriodicDist<A, K, M>> pol(k, b.radius(radius0, qi), pd);
      warp_periodic_query<A, K, M>(tv, q, box.v, pol, lane, st);
      pol.write(qi, out_d, out_i, out_c, false, lane);
    }
    if (stats && lane == 0) add_stats(stats, st);
  });
}

template <typename A, int K, typename M, bool EXCL>
__global__ void __launch_bounds__(256) k_periodic_within_count(
    TreeView<A> tv0, Batch<A> b, BoxArg<A, K> box, A radius0, uint64_t* __restrict__ counts,
    unsigned long long* __restrict__ stats) {
  const int lane = threadIdx.x & 31;
  PeriodicDist<A, K, M> pd;
#pragma unroll
  for (int d = 0; d < K; ++d) pd.box[d] = box.v[d];
  for_each_query_warp(b, [&](uint64_t qi) {
    const TreeView<A> tv = b.tree(tv0, qi);
    A q[K];
    b.query(qi, q);
    WithinCountPolicy<A, K, M, EXCL, PeriodicDist<A, K, M>> pol(b.radius(radius0, qi), pd);
    TravStats st;
    warp_periodic_query<A, K, M>(tv, q, box.v, pol, lane, st);
    if (lane == 0) counts[qi] = pol.count;
    if (stats && lane == 0) add_stats(stats, st);
  });
}

template <typename A, int K, typename M, bool EXCL>
__global__ void __launch_bounds__(256) k_periodic_within_fill(
    TreeView<A> tv0, Batch<A> b, BoxArg<A, K> box, A radius0, const uint64_t* __restrict__ offsets,
    uint64_t capacity, A* __restrict__ out_d, uint32_t* __restrict__ out_i,
    int* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  PeriodicDist<A, K, M> pd;
#pragma unroll
  for (int d = 0; d < K; ++d) pd.box[d] = box.v[d];
  for_each_query_warp(b, [&](uint64_t qi) {
    const uint64_t o = offsets[qi];
    const uint64_t end = offsets[qi + 1] < capacity ? offsets[qi + 1] : capacity;
    if (end <= o) return;
    const TreeView<A> tv = b.tree(tv0, qi);
    A q[K];
    b.query(qi, q);
    WithinFillPolicy<A, K, M, EXCL, PeriodicDist<A, K, M>> pol(b.radius(radius0, qi), end - o,
                                                                out_d + o, out_i + o, pd);
    TravStats st;
    warp_periodic_query<A, K, M>(tv, q, box.v, pol, lane, st);
    if (lane == 0 && status && pol.count != offsets[qi + 1] - o) atomicExch(status, 6);
  });
}

// Segments of at most 32 hits: one warp, bitonic network on (distance, position)
// so equal distances keep traversal order (a stable sort, as Vec::sort).
template <typename A>
__device__ __forceinline__ bool key_less(A da, uint32_t pa, A db, uint32_t pb) {
  return da < db || (da == db && pa < pb);
}

// Stable sort of one segment of n <= N hits by its own thread: the segment is
// loaded into registers (padding +inf after it), insertion-sorted by a fully
// unrolled network of adjacent compare-swaps that swap only strictly greater
// keys (so equal keys keep their order and padding stays behind), and written
// back.
template <typename A, int N>
__device__ __forceinline__ void small_segment_sort(A* __restrict__ d, uint32_t* __restrict__ it,
                                                   uint32_t n) {
  A kd[N];
  uint32_t kv[N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    kd[j] = uint32_t(j) < n ? d[j] : inf_of<A>();
    kv[j] = uint32_t(j) < n ? it[j] : 0u;
  }
#pragma unroll
  for (int a = 1; a < N; ++a) {
#pragma unroll
    for (int j = a; j > 0; --j) {
      const bool sw = kd[j - 1] > kd[j];
      const A td = kd[j - 1];
      const uint32_t tv = kv[j - 1];
      kd[j - 1] = sw ? kd[j] : td;
      kv[j - 1] = sw ? kv[j] : tv;
      kd[j] = sw ? td : kd[j];
      kv[j] = sw ? tv : kv[j];
    }
  }
#pragma unroll
  for (int j = 0; j < N; ++j)
    if (uint32_t(j) < n) {
      d[j] = kd[j];
      it[j] = kv[j];
    }
}

// Segments of up to 32 hits.  A warp takes 32 segments at a time (lane l
// reads segment base + l's bounds, coalesced): segments of 2..kThreadSort
// hits are sorted in registers by their own lane (small_segment_sort), and
// the warp then bitonic-sorts its segments of
// kThreadSort+1..32 hits one after another on (key, position).
template <typename A>
__global__ void __launch_bounds__(256) k_seg_sort_warp(const uint64_t* __restrict__ offsets,
                                                       uint64_t nq, uint64_t capacity,
                                                       A* __restrict__ d,
                                                       uint32_t* __restrict__ it) {
  constexpr uint64_t kThreadSort = 8;
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t base = warp * 32; base < nq; base += nwarps * 32) {
    const uint64_t s = base + lane;
    uint64_t o = 0, n = 0;
    if (s < nq) {
      o = min(offsets[s], capacity);
      n = min(offsets[s + 1], capacity) - o;
    }
    if (n >= 2 && n <= 4) {
      small_segment_sort<A, 4>(d + o, it + o, uint32_t(n));
    } else if (n > 4 && n <= kThreadSort) {
      small_segment_sort<A, kThreadSort>(d + o, it + o, uint32_t(n));
    }
    for (unsigned big = __ballot_sync(FULL, n > kThreadSort && n <= 32); big; big &= big - 1) {
      const int src = __ffs(big) - 1;
      const uint64_t so = __shfl_sync(FULL, (unsigned long long)o, src);
      const uint32_t sn = uint32_t(__shfl_sync(FULL, (unsigned long long)n, src));
      A kd = inf_of<A>();
      uint32_t kp = 0xffffffffu, kv = 0;
      if (uint32_t(lane) < sn) { kd = d[so + lane]; kv = it[so + lane]; kp = lane; }
#pragma unroll
      for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          const A od = __shfl_xor_sync(FULL, kd, stride);
          const uint32_t op = __shfl_xor_sync(FULL, kp, stride);
          const uint32_t ov = __shfl_xor_sync(FULL, kv, stride);
          const bool up = ((lane & size) == 0);
          const bool lower = (lane & stride) == 0;
          // lower lane keeps the min when ascending
          const bool other_less = key_less(od, op, kd, kp);
          const bool take = lower ? (up ? other_less : !other_less) : (up ? !other_less : other_less);
          if (take && !(od == kd && op == kp)) { kd = od; kp = op; kv = ov; }
        }
      }
      if (uint32_t(lane) < sn) { d[so + lane] = kd; it[so + lane] = kv; }
    }
  }
}

// Stable merge step (merge path): out[lo..hi) from runs a[0..na) and b[0..nb),
// ties taken from `a` first.
template <typename A>
__device__ __forceinline__ void merge_range(const A* ad, const uint32_t* ai, uint32_t na,
                                            const A* bd, const uint32_t* bi, uint32_t nb,
                                            A* od, uint32_t* oi, uint32_t lo, uint32_t hi) {
  if (lo >= hi) return;
  uint32_t l = lo > nb ? lo - nb : 0, h = lo < na ? lo : na;
  while (l < h) {
    const uint32_t mid = (l + h) >> 1;
    if (!(bd[lo - mid - 1] < ad[mid])) l = mid + 1;  // ad[mid] <= bd[...]: a first
    else h = mid;
  }
  uint32_t x = l, y = lo - l;
  for (uint32_t o = lo; o < hi; ++o) {
    bool take_a = x < na && (y >= nb || !(bd[y] < ad[x]));
    if (take_a) { od[o] = ad[x]; oi[o] = ai[x]; ++x; }
    else { od[o] = bd[y]; oi[o] = bi[y]; ++y; }
  }
}

// Bottom-up stable merge sort of one segment by the whole block, ping-ponging
// between (d0, i0) and (d1, i1).  Returns true if the result ended in (d1, i1).
template <typename A>
__device__ bool block_merge_sort(A* d0, uint32_t* i0, A* d1, uint32_t* i1, uint32_t n) {
  bool in1 = false;
  for (uint32_t width = 1; width < n; width <<= 1) {
    A* sd = in1 ? d1 : d0;
    uint32_t* si = in1 ? i1 : i0;
    A* td = in1 ? d0 : d1;
    uint32_t* ti = in1 ? i0 : i1;
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = threadIdx.x * per;
    const uint32_t hi = min(n, lo + per);
    // each thread's output range may span several run pairs
    uint32_t o = lo;
    while (o < hi) {
      const uint32_t pair = o / (2 * width);
      const uint32_t start = pair * 2 * width;
      const uint32_t mid = min(n, start + width);
      const uint32_t end = min(n, start + 2 * width);
      const uint32_t stop = min(hi, end);
      merge_range<A>(sd + start, si + start, mid - start, sd + mid, si + mid, end - mid,
                     td + start, ti + start, o - start, stop - start);
      o = stop;
    }
    __syncthreads();
    in1 = !in1;
  }
  return in1;
}

// Segments longer than 32: one block per group of 256 segments; each long
// segment is sorted by the whole block in shared memory when it fits, else in
// global memory with `scratch` as the second buffer.
template <typename A>
__global__ void __launch_bounds__(256) k_seg_sort_block(const uint64_t* __restrict__ offsets,
                                                        uint64_t nq, uint64_t capacity,
                                                        A* __restrict__ d,
                                                        uint32_t* __restrict__ it,
                                                        A* __restrict__ scratch_d,
                                                        uint32_t* __restrict__ scratch_i,
                                                        uint32_t smem_cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t list[256];
  __shared__ uint32_t list_n;
  const uint64_t first = uint64_t(blockIdx.x) * 256;
  if (threadIdx.x == 0) list_n = 0;
  __syncthreads();
  {
    const uint64_t s = first + threadIdx.x;
    if (s < nq) {
      const uint64_t n = min(offsets[s + 1], capacity) - min(offsets[s], capacity);
      if (n > 32) list[atomicAdd(&list_n, 1u)] = uint32_t(threadIdx.x);
    }
  }
  __syncthreads();
  const uint32_t cnt = list_n;
  A* sd0 = reinterpret_cast<A*>(smem_raw);
  A* sd1 = sd0 + smem_cap;
  uint32_t* si0 = reinterpret_cast<uint32_t*>(sd1 + smem_cap);
  uint32_t* si1 = si0 + smem_cap;
  for (uint32_t j = 0; j < cnt; ++j) {
    const uint64_t s = first + list[j];
    const uint64_t o = min(offsets[s], capacity);
    const uint32_t n = uint32_t(min(offsets[s + 1], capacity) - o);
    if (n <= smem_cap) {
      for (uint32_t x = threadIdx.x; x < n; x += blockDim.x) { sd0[x] = d[o + x]; si0[x] = it[o + x]; }
      __syncthreads();
      const bool in1 = block_merge_sort<A>(sd0, si0, sd1, si1, n);
      const A* rd = in1 ? sd1 : sd0;
      const uint32_t* ri = in1 ? si1 : si0;
      for (uint32_t x = threadIdx.x; x < n; x += blockDim.x) { d[o + x] = rd[x]; it[o + x] = ri[x]; }
      __syncthreads();
    } else {
      const bool in1 = block_merge_sort<A>(d + o, it + o, scratch_d + o, scratch_i + o, n);
      if (in1) {
        for (uint32_t x = threadIdx.x; x < n; x += blockDim.x) {
          d[o + x] = scratch_d[o + x];
          it[o + x] = scratch_i[o + x];
        }
      }
      __syncthreads();
    }
  }
}

}  // namespace kgpu

namespace kgpu {

// ---------------------------------------------------------------------------
// Leaf-bucketed processing order (KGPU_FLAG_SPATIAL_ORDER): each query's
// straight-descent leaf (traits/stem_strategy.rs:182-200) is its bucket; a
// counting sort over buckets gives an order in which neighbouring threads
// walk the same stems and leaves.  Results do not depend on the order.
// ---------------------------------------------------------------------------
template <typename A, int K>
__global__ void __launch_bounds__(256) k_leaf_histogram(TreeView<A> tv0, Batch<A> b,
                                                        const uint64_t* __restrict__ leaf_base,
                                                        uint32_t* __restrict__ leaf_of,
                                                        unsigned long long* __restrict__ counts) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < b.nq;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const TreeView<A> tv = b.tree(tv0, i);
    A q[K];
    b.query(i, q);
    uint64_t l = tv.leaf_count > 1 ? straight_leaf<A, K>(tv, q) : 0u;
    if (leaf_base) l += b.tree_of[i] < b.n_trees ? leaf_base[b.tree_of[i]] : 0u;
    leaf_of[i] = uint32_t(l);
    atomicAdd(counts + l, 1ull);
  }
}

static __global__ void __launch_bounds__(256) k_leaf_scatter(const uint32_t* __restrict__ leaf_of,
                                                      uint64_t nq,
                                                      unsigned long long* __restrict__ cursor,
                                                      uint32_t* __restrict__ order) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nq;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const unsigned long long pos = atomicAdd(cursor + leaf_of[i], 1ull);
    order[pos] = uint32_t(i);
  }
}

}  // namespace kgpu
