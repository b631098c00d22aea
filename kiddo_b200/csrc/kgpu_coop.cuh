// kgpu_coop.cuh — warp-cooperative leaf scans for the thread-per-query engine.
//
// Each thread walks its own query's tree (ThreadWalk, the reference's DFS).
// When the lanes of a warp have reached their next leaves, the warp scans
// those leaves one after another, all 32 lanes on one leaf: lane p takes
// point p, so the coordinate columns of a 32-point tile load as one coalesced
// 128-byte row per axis.  A ballot picks the points that pass the leaf-start
// filter, and the candidates are then applied in arrival order (lane order)
// to the owner's result list, which sits one entry per lane for the scan:
// an insertion is one ballot (its position) and one shuffle up (the shift).
//
// Each family keeps the sequential semantics of its reference collector:
// best_n_within the n smallest by (item, arrival) (kd_tree/query/
// best_n_within.rs:88-196), within appends hits in arrival order
// (kd_tree/query/within.rs:18-41).  (For nearest_n the per-candidate
// insertions are paid per candidate while a per-thread scan pays per point;
// nearest_n scans per thread unless KGPU_FLAG_ENGINE_COOP asks for this form,
// and nearest_one always scans per thread.)
#pragma once

#include "kgpu_device.cuh"
#include "kgpu_thread.cuh"

namespace kgpu {

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
  return __shfl_sync(FULL, static_cast<unsigned long long>(v), src);
}

__device__ __forceinline__ unsigned lanes_below() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// The leaf one lane reached, as the whole warp sees it while scanning it.
template <typename A, int K>
struct CoopLeaf {
  const uint8_t* base;
  uint32_t len;
  A q[K];
};

template <typename A, int K>
__device__ __forceinline__ CoopLeaf<A, K> coop_leaf(int o, const uint8_t* base, uint32_t len,
                                                    const A (&q)[K]) {
  CoopLeaf<A, K> L;
  L.base = reinterpret_cast<const uint8_t*>(shfl64(reinterpret_cast<uint64_t>(base), o));
  L.len = shfl(len, o);
#pragma unroll
  for (int d = 0; d < K; ++d) L.q[d] = shfl(q[d], o);
  return L;
}

// Distance (Cartesian or periodic functor) from the owner's query to point
// p (< len) of the leaf.
template <typename A, int K, typename Dist>
__device__ __forceinline__ A coop_point(const CoopLeaf<A, K>& L, uint32_t p, uint32_t& item,
                                        const Dist& dist) {
  A c[K];
  load_point<A, K>(L.base, L.len, p, c, item);
  return dist(c, L.q);
}

// ---------------------------------------------------------------------------
// best_n_within: the n smallest items among the hits, by (item, arrival);
// the leaf filter drops items >= the list's last item when the leaf starts
// with a full list (leaf_view_chunked/best_n_within/fallback.rs:40-104).
// ---------------------------------------------------------------------------
template <typename A, int K, typename M, bool kExclusive>
struct CBestN {
  static constexpr bool kPruneOnEqual = kExclusive;
  A* __restrict__ wd;
  uint32_t* __restrict__ wi;
  int k;
  int n;
  A radius;
  uint32_t last;  // the list's last item once full
  __device__ CBestN(A* d, uint32_t* i, uint32_t*, int k_, A r)
      : wd(d), wi(i), k(k_), n(0), radius(r), last(0) {}
  __device__ __forceinline__ void reset(A r) { n = 0; radius = r; last = 0; }
  __device__ __forceinline__ A max_dist() const { return radius; }
  __device__ __forceinline__ bool unbounded_start() const { return false; }

  __device__ __forceinline__ void leaf(int o, uint64_t, const CoopLeaf<A, K>& L, int lane) {
    int nn = __shfl_sync(FULL, n, o);
    uint32_t lk = shfl(last, o);
    const A orad = shfl(radius, o);
    const bool full_at_entry = nn == k;
    const uint32_t thr_item = lk;
    A* ld = wd + o * k;
    uint32_t* li = wi + o * k;
    A Ld = A(0);
    uint32_t Li = 0xffffffffu;
    bool loaded = false;
    for (uint32_t c0 = 0; c0 < L.len; c0 += 32) {
      const uint32_t p = c0 + lane;
      A d = A(0);
      uint32_t it = 0;
      bool pass = false;
      if (p < L.len) {
        d = coop_point<A, K>(L, p, it, CartesianDist<A, K, M>());
        pass = (kExclusive ? (d < orad) : (d <= orad)) && !(full_at_entry && it >= thr_item) &&
               (nn < k || it < lk);
      }
      unsigned m = __ballot_sync(FULL, pass);
      if (m && !loaded) {
        if (lane < nn) {
          Ld = ld[lane];
          Li = li[lane];
        }
        loaded = true;
      }
      while (m) {
        const int c = __ffs(m) - 1;
        m &= m - 1;
        const A dc = shfl(d, c);
        const uint32_t ic = shfl(it, c);
        if (nn == k && !(ic < lk)) continue;
        const int pos = __popc(__ballot_sync(FULL, lane < nn && Li <= ic));
        const A ud = __shfl_up_sync(FULL, Ld, 1);
        const uint32_t ui = __shfl_up_sync(FULL, Li, 1);
        if (lane > pos) {
          Ld = ud;
          Li = ui;
        } else if (lane == pos) {
          Ld = dc;
          Li = ic;
        }
        if (nn < k) ++nn;
        if (nn == k) lk = shfl(Li, k - 1);
      }
    }
    if (loaded && lane < nn) {
      ld[lane] = Ld;
      li[lane] = Li;
    }
    if (lane == o) {
      n = nn;
      last = lk;
    }
  }

  __device__ __forceinline__ void finish(int o, uint64_t qi, int lane, A* __restrict__ out_d,
                                         uint32_t* __restrict__ out_i,
                                         uint32_t* __restrict__ out_c) const {
    const int on = __shfl_sync(FULL, n, o);
    if (lane < k) {
      const bool h = lane < on;
      out_d[qi * k + lane] = h ? wd[o * k + lane] : inf_of<A>();
      out_i[qi * k + lane] = h ? wi[o * k + lane] : 0xffffffffu;
    }
    if (lane == 0 && out_c) out_c[qi] = uint32_t(on);
  }
};

// ---------------------------------------------------------------------------
// nearest_n / nearest_n().within, sorted output: the k smallest by (distance,
// arrival) (ThresholdVecResultCollection, results/result_collection.rs:
// 136-215), kept sorted in the query's own output row, which a leaf scan
// reads and writes one entry per lane.  A candidate goes after every held
// entry of distance <= its own (those arrived first); once the list is full
// it must beat the last entry, which it evicts.
// ---------------------------------------------------------------------------
template <typename A, int K, typename M, bool kExclusive, typename Dist>
struct CNearestNRow {
  static constexpr bool kPruneOnEqual = kExclusive;
  A* __restrict__ out_d;
  uint32_t* __restrict__ out_i;
  int k;
  int n;
  A radius, kth;
  Dist dist;
  __device__ CNearestNRow(A* d, uint32_t* i, int k_, Dist ds)
      : out_d(d), out_i(i), k(k_), n(0), radius(A(0)), kth(inf_of<A>()), dist(ds) {}
  __device__ __forceinline__ void reset(A r) { n = 0; radius = r; kth = inf_of<A>(); }
  __device__ __forceinline__ A max_dist() const { return (n == k && kth < radius) ? kth : radius; }
  __device__ __forceinline__ bool unbounded_start() const { return radius == inf_of<A>(); }

  // Chunks with this many candidates are merged at once instead of inserted
  // one by one.
#ifndef KGPU_COOP_MERGE_FROM
#define KGPU_COOP_MERGE_FROM 6
#endif
  static constexpr int kMergeFrom = KGPU_COOP_MERGE_FROM;

  // All candidates of a chunk at once.  The candidates are bitonic-sorted by
  // (distance, lane) -- lane order is arrival order -- with non-candidates
  // behind them; then every held entry and every candidate learns its place in
  // the merged sequence by a binary search of the other sorted sequence (held
  // entries ahead of candidates of equal distance, since they arrived first),
  // the first k are written to the row, and the row is read back.  This is
  // the list the one-by-one inserts would leave: the k smallest by (distance,
  // arrival) of the held entries and the candidates.
  __device__ __forceinline__ void merge_chunk(bool pass, A d, uint32_t it, int cnt, int& nn, A& kk,
                                              A& Ld, uint32_t& Li, A* __restrict__ ld,
                                              uint32_t* __restrict__ li, int lane) const {
    A sd = d;
    uint32_t si = it;
    uint32_t tag = (pass ? 0u : 32u) | uint32_t(lane);  // non-candidates sort last
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        const A od = __shfl_xor_sync(FULL, sd, stride);
        const uint32_t ot = __shfl_xor_sync(FULL, tag, stride);
        const uint32_t oi = __shfl_xor_sync(FULL, si, stride);
        const bool up = (lane & size) == 0;
        const bool lower = (lane & stride) == 0;
        // key order: candidates first, then distance, then lane
        const bool other_less =
            (ot >> 5) != (tag >> 5) ? (ot >> 5) < (tag >> 5) : (od < sd || (od == sd && ot < tag));
        const bool take = lower ? (up ? other_less : !other_less) : (up ? !other_less : other_less);
        if (take) {
          sd = od;
          tag = ot;
          si = oi;
        }
      }
    }
    // rank of a held entry among the candidates (strictly closer ones) and of
    // a candidate among the held entries (not farther ones)
    int lo = 0, hi = cnt;
    int lo2 = 0, hi2 = nn;
#pragma unroll
    for (int step = 0; step < 6; ++step) {
      const int mid = (lo + hi) >> 1;
      const A v = shfl(sd, mid & 31);
      if (lo < hi) {
        if (v < Ld) lo = mid + 1;
        else hi = mid;
      }
      const int mid2 = (lo2 + hi2) >> 1;
      const A v2 = shfl(Ld, mid2 & 31);
      if (lo2 < hi2) {
        if (v2 <= sd) lo2 = mid2 + 1;
        else hi2 = mid2;
      }
    }
    const int pos_held = lane + lo, pos_cand = lane + lo2;
    if (lane < nn && pos_held < k) {
      ld[pos_held] = Ld;
      li[pos_held] = Li;
    }
    if (lane < cnt && pos_cand < k) {
      ld[pos_cand] = sd;
      li[pos_cand] = si;
    }
    __syncwarp();
    nn = nn + cnt < k ? nn + cnt : k;
    Ld = inf_of<A>();
    Li = 0;
    if (lane < nn) {
      Ld = ld[lane];
      Li = li[lane];
    }
    if (nn == k) kk = shfl(Ld, k - 1);
    __syncwarp();
  }

  __device__ __forceinline__ void leaf(int o, uint64_t qo, const CoopLeaf<A, K>& L, int lane) {
    int nn = __shfl_sync(FULL, n, o);
    A kk = shfl(kth, o);
    const A orad = shfl(radius, o);
    const A bound = (nn == k && kk < orad) ? kk : orad;  // max_dist() at leaf start
    A* ld = out_d + qo * uint64_t(k);
    uint32_t* li = out_i + qo * uint64_t(k);
    A Ld = inf_of<A>();
    uint32_t Li = 0;
    bool loaded = false;
    for (uint32_t c0 = 0; c0 < L.len; c0 += 32) {
      const uint32_t p = c0 + lane;
      A d = inf_of<A>();
      uint32_t it = 0;
      bool pass = false;
      if (p < L.len) {
        d = coop_point<A, K>(L, p, it, dist);
        pass = (kExclusive ? (d < bound) : (d <= bound)) && (nn < k || d < kk);
      }
      unsigned m = __ballot_sync(FULL, pass);
      if (m && !loaded) {
        if (lane < nn) {
          Ld = ld[lane];
          Li = li[lane];
        }
        loaded = true;
      }
      const int cnt = __popc(m);
      if (cnt >= kMergeFrom) {
        merge_chunk(pass, d, it, cnt, nn, kk, Ld, Li, ld, li, lane);
        continue;
      }
      while (m) {
        const int c = __ffs(m) - 1;
        m &= m - 1;
        const A dc = shfl(d, c);
        const uint32_t ic = shfl(it, c);
        if (nn == k && !(dc < kk)) continue;
        const int pos = __popc(__ballot_sync(FULL, lane < nn && Ld <= dc));
        const A ud = __shfl_up_sync(FULL, Ld, 1);
        const uint32_t ui = __shfl_up_sync(FULL, Li, 1);
        if (lane > pos) {
          Ld = ud;
          Li = ui;
        } else if (lane == pos) {
          Ld = dc;
          Li = ic;
        }
        if (nn < k) ++nn;
        if (nn == k) kk = shfl(Ld, k - 1);
      }
    }
    if (loaded && lane < nn) {
      ld[lane] = Ld;
      li[lane] = Li;
    }
    if (lane == o) {
      n = nn;
      kth = kk;
    }
  }

  // The held entries are already in place; the rest of the row is
  // (+inf, u32::MAX).
  __device__ __forceinline__ void finish(int o, uint64_t qo, int lane,
                                         uint32_t* __restrict__ out_c) const {
    const int on = __shfl_sync(FULL, n, o);
    if (lane >= on && lane < k) {
      out_d[qo * uint64_t(k) + lane] = inf_of<A>();
      out_i[qo * uint64_t(k) + lane] = 0xffffffffu;
    }
    if (lane == 0 && out_c) out_c[qo] = uint32_t(on);
  }
};

// ---------------------------------------------------------------------------
// Lists of any length, kept in the query's own output row: nearest_n (the k
// smallest by (distance, arrival), the reference's ThresholdVec or, above its
// range, BinaryHeap collector with the same distance multiset,
// results/result_collection.rs:136-215, 365-560) or best_n_within (`BEST`, a
// run-time choice: the n smallest items by (item, arrival),
// result_collection.rs:463-560).  A leaf is
// scanned by the whole warp for its owner; each candidate, in leaf order, finds
// its place with one ballot per 32 held entries (after the entries whose key is
// not above its own, which arrived first) and the entries behind it move up
// one place, 32 at a time from the top; a full list drops its last entry.
// Output rows are always sorted (by distance, or by item for best_n).
// ---------------------------------------------------------------------------
template <typename A, int K, typename M, bool kExclusive, typename Dist>
struct CRowList {
  static constexpr bool kPruneOnEqual = kExclusive;
  bool BEST;  // best_n_within (by item) rather than nearest_n (by distance)
  A* __restrict__ out_d;
  uint32_t* __restrict__ out_i;
  int k;
  int n;
  A radius, kth;
  uint32_t last;  // best_n: the last item once full
  Dist dist;
  __device__ CRowList(bool best, A* d, uint32_t* i, int k_, Dist ds)
      : BEST(best), out_d(d), out_i(i), k(k_), n(0), radius(A(0)), kth(inf_of<A>()), last(0),
        dist(ds) {}
  __device__ __forceinline__ void reset(A r) {
    n = 0;
    radius = r;
    kth = inf_of<A>();
    last = 0;
  }
  __device__ __forceinline__ A max_dist() const {
    if (BEST) return radius;
    return (n == k && kth < radius) ? kth : radius;
  }
  __device__ __forceinline__ bool unbounded_start() const {
    return !BEST && radius == inf_of<A>();
  }

  __device__ __forceinline__ void leaf(int o, uint64_t qo, const CoopLeaf<A, K>& L, int lane) {
    int nn = __shfl_sync(FULL, n, o);
    A kk = shfl(kth, o);
    uint32_t lk = shfl(last, o);
    const A orad = shfl(radius, o);
    const bool full_at_entry = nn == k;
    const uint32_t thr_item = lk;
    // the leaf filter's bound: max_dist() at leaf start
    const A bound = (!BEST && nn == k && kk < orad) ? kk : orad;
    A* rd = out_d + qo * uint64_t(k);
    uint32_t* ri = out_i + qo * uint64_t(k);
    for (uint32_t c0 = 0; c0 < L.len; c0 += 32) {
      const uint32_t p = c0 + lane;
      A d = inf_of<A>();
      uint32_t it = 0;
      bool pass = false;
      if (p < L.len) {
        d = coop_point<A, K>(L, p, it, dist);
        pass = kExclusive ? (d < bound) : (d <= bound);
        if (BEST) pass = pass && !(full_at_entry && it >= thr_item) && (nn < k || it < lk);
        else pass = pass && (nn < k || d < kk);
      }
      unsigned m = __ballot_sync(FULL, pass);
      while (m) {
        const int c = __ffs(m) - 1;
        m &= m - 1;
        const A dc = shfl(d, c);
        const uint32_t ic = shfl(it, c);
        if (nn == k && (BEST ? !(ic < lk) : !(dc < kk))) continue;
        int pos = 0;  // held entries whose key is not above the candidate's
        for (int j0 = 0; j0 < nn; j0 += 32) {
          const int j = j0 + lane;
          bool le = false;
          if (j < nn) le = BEST ? !(ri[j] > ic) : !(rd[j] > dc);
          pos += __popc(__ballot_sync(FULL, le));
        }
        const int top = nn < k ? nn - 1 : k - 2;  // entries pos..top move up one
        for (int j0 = top & ~31; top >= pos && j0 >= (pos & ~31); j0 -= 32) {
          const int j = j0 + lane;
          const bool mv = j >= pos && j <= top;
          A vd = A(0);
          uint32_t vi = 0;
          if (mv) {
            vd = rd[j];
            vi = ri[j];
          }
          __syncwarp();
          if (mv) {
            rd[j + 1] = vd;
            ri[j + 1] = vi;
          }
          __syncwarp();
        }
        if (lane == 0) {
          rd[pos] = dc;
          ri[pos] = ic;
        }
        __syncwarp();
        if (nn < k) ++nn;
        if (nn == k) {
          if (BEST) lk = ri[k - 1];
          else kk = rd[k - 1];
        }
      }
    }
    if (lane == o) {
      n = nn;
      kth = kk;
      last = lk;
    }
  }

  // The held entries are in place; the rest of the row is (+inf, u32::MAX).
  __device__ __forceinline__ void finish(int o, uint64_t qo, int lane,
                                         uint32_t* __restrict__ out_c) const {
    const int on = __shfl_sync(FULL, n, o);
    for (int j = on + lane; j < k; j += 32) {
      out_d[qo * uint64_t(k) + j] = inf_of<A>();
      out_i[qo * uint64_t(k) + j] = 0xffffffffu;
    }
    if (lane == 0 && out_c) out_c[qo] = uint32_t(on);
  }
};

// ---------------------------------------------------------------------------
// within: counting pass (no output) or filling pass (hits written in arrival
// order into the query's CSR segment, `cap` long); a leaf's hits are one
// coalesced store.
// ---------------------------------------------------------------------------
template <typename A, int K, typename M, bool kExclusive, typename Dist = CartesianDist<A, K, M>>
struct CWithin {
  static constexpr bool kPruneOnEqual = kExclusive;
  A radius;
  uint64_t count;
  uint64_t cap;
  A* out_d;
  uint32_t* out_i;
  Dist dist;
  __device__ explicit CWithin(Dist ds = Dist())
      : radius(A(0)), count(0), cap(0), out_d(nullptr), out_i(nullptr), dist(ds) {}
  __device__ __forceinline__ A max_dist() const { return radius; }
  __device__ __forceinline__ bool unbounded_start() const { return radius == inf_of<A>(); }

  __device__ __forceinline__ void leaf(int o, uint64_t, const CoopLeaf<A, K>& L, int lane) {
    leaf(o, L, lane);
  }
  __device__ __forceinline__ void leaf(int o, const CoopLeaf<A, K>& L, int lane) {
    uint64_t cnt = shfl64(count, o);
    const uint64_t ocap = shfl64(cap, o);
    A* od = reinterpret_cast<A*>(shfl64(reinterpret_cast<uint64_t>(out_d), o));
    uint32_t* oi = reinterpret_cast<uint32_t*>(shfl64(reinterpret_cast<uint64_t>(out_i), o));
    const A orad = shfl(radius, o);
    for (uint32_t c0 = 0; c0 < L.len; c0 += 32) {
      const uint32_t p = c0 + lane;
      A d = A(0);
      uint32_t it = 0;
      bool pass = false;
      if (p < L.len) {
        d = coop_point<A, K>(L, p, it, dist);
        pass = kExclusive ? (d < orad) : (d <= orad);
      }
      const unsigned m = __ballot_sync(FULL, pass);
      if (od && pass) {
        const uint64_t w = cnt + uint64_t(__popc(m & lanes_below()));
        if (w < ocap) {
          od[w] = d;
          oi[w] = it;
        }
      }
      cnt += uint64_t(__popc(m));
    }
    if (lane == o) count = cnt;
  }
};

}  // namespace kgpu
