// kgpu_device.cuh — device building blocks of the query engine (sm_100a).
//
// One warp answers one query.  Every lane keeps an identical copy of the
// query's scalar traversal state (stem index, level, per-axis offsets, rd,
// the pending-far bitmask) so the descent needs no shuffles; the per-level
// continuation records of kiddo's arithmetic traversal
// (kd_tree/orchestrator/mod.rs:388-603: restore frame {old_off, has_far} and
// far frame {stem, far_off, rd}) live in registers of the lane whose index is
// the level ("per-lane register stacks").  The 32 lanes then scan a leaf's
// points side by side: lane i reads point i of the VecOfArenas tile, so the
// column loads of a 32-wide tile are one coalesced transaction per axis.
//
// All distance and rectangle-distance arithmetic uses the explicitly rounded
// intrinsics (__fadd_rn/__fsub_rn/__fmul_rn and the double forms), in the
// reference's order, so no multiply-add is ever contracted; the translation
// unit is also compiled with -fmad=false.
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace kgpu {

constexpr unsigned FULL = 0xffffffffu;

// ---------------------------------------------------------------------------
// exactly rounded scalar helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float abs_val(float a) { return fabsf(a); }
__device__ __forceinline__ double abs_val(double a) { return fabs(a); }

template <typename A> __device__ __forceinline__ A inf_of();
template <> __device__ __forceinline__ float inf_of<float>() { return __int_as_float(0x7f800000); }
template <> __device__ __forceinline__ double inf_of<double>() {
  return __longlong_as_double(0x7ff0000000000000ll);
}

__device__ __forceinline__ float shfl(float v, int src) { return __shfl_sync(FULL, v, src); }
__device__ __forceinline__ double shfl(double v, int src) { return __shfl_sync(FULL, v, src); }
__device__ __forceinline__ uint32_t shfl(uint32_t v, int src) { return __shfl_sync(FULL, v, src); }
__device__ __forceinline__ float shfl_up(float v, int d) { return __shfl_up_sync(FULL, v, d); }
__device__ __forceinline__ double shfl_up(double v, int d) { return __shfl_up_sync(FULL, v, d); }
__device__ __forceinline__ uint32_t shfl_up(uint32_t v, int d) { return __shfl_up_sync(FULL, v, d); }

// ---------------------------------------------------------------------------
// Metrics (dist/distance_metric_core.rs:12-105)
// ---------------------------------------------------------------------------
// Element d of a small register array, read and written without local memory.
template <typename A, int K>
__device__ __forceinline__ A sel(const A (&v)[K], int d) {
  A r = v[0];
#pragma unroll
  for (int j = 1; j < K; ++j)
    if (d == j) r = v[j];
  return r;
}
template <typename A, int K>
__device__ __forceinline__ void put(A (&v)[K], int d, A x) {
#pragma unroll
  for (int j = 0; j < K; ++j)
    if (d == j) v[j] = x;
}

// Every metric runs periodic queries (periodic.rs is generic over the
// metric: combine_component over min-image components, and the metric's own
// rect_dist_after_update over the interval offsets).
// The additive metrics: combine_component is acc + component, and the
// rectangle distance after one axis offset changes is the O(1) update of
// rect() (distance_metric_core.rs:38-44, 86-96).  kPacked marks the two whose
// point pairs take the packed f32x2 subtract/multiply path.
template <typename Self>
struct Additive {
  static constexpr bool kPeriodic = true;
  static constexpr bool kAdditive = true;
  static constexpr bool kPacked = false;
  template <typename A> __device__ __forceinline__ static A combine(A acc, A comp) {
    return add_rn(acc, comp);
  }
  template <typename A, int K>
  __device__ __forceinline__ static A rect_k(A rd, const A (&off)[K], int dim, A new_off) {
    return Self::template rect<A>(rd, sel(off, dim), new_off);
  }
};

struct SqEuclidean : Additive<SqEuclidean> {
  static constexpr bool kPacked = true;
  // dist1(a, b) = (a - b)^2   (dist/squared_euclidean/mod.rs:35-38)
  template <typename A> __device__ __forceinline__ static A dist1(A a, A b) {
    const A d = sub_rn(a, b);
    return mul_rn(d, d);
  }
  // (rd - dist1(old, 0)) + dist1(new, 0)   (distance_metric_core.rs:86-96)
  template <typename A> __device__ __forceinline__ static A rect(A rd, A old_off, A new_off) {
    return add_rn(sub_rn(rd, mul_rn(old_off, old_off)), mul_rn(new_off, new_off));
  }
};

struct Manhattan : Additive<Manhattan> {
  static constexpr bool kPacked = true;
  // |a - b|   (dist/manhattan/mod.rs:35-38)
  template <typename A> __device__ __forceinline__ static A dist1(A a, A b) {
    return abs_val(sub_rn(a, b));
  }
  // (rd - old) + new   (dist/manhattan/mod.rs:40-48)
  template <typename A> __device__ __forceinline__ static A rect(A rd, A old_off, A new_off) {
    return add_rn(sub_rn(rd, old_off), new_off);
  }
};

// Minkowski<P> (dist/minkowski/mod.rs:19-58): dist1 = |a - b|.powi(P), summed
// without the final root.  Rust's powi is llvm.powi, expanded by binary
// exponentiation (result times the running square, low bit first), so
// x^3 = x * (x * x) and x^4 = (x * x) * (x * x), each product rounded.  P = 3
// and 4.
template <int P>
struct Minkowski : Additive<Minkowski<P>> {
  static_assert(P == 3 || P == 4, "Minkowski<3> and Minkowski<4>");
  template <typename A> __device__ __forceinline__ static A dist1(A a, A b) {
    const A x = abs_val(sub_rn(a, b));
    const A x2 = mul_rn(x, x);
    return P == 3 ? mul_rn(x, x2) : mul_rn(x2, x2);
  }
  template <typename A> __device__ __forceinline__ static A rect(A rd, A old_off, A new_off) {
    return add_rn(sub_rn(rd, dist1(old_off, A(0))), dist1(new_off, A(0)));
  }
};

// Chebyshev / L-infinity (dist/chebyshev/mod.rs:19-59): dist1 = |a - b|,
// combine_component keeps the larger value (a component that is not greater,
// NaN included, leaves the accumulator as it is), and the rectangle distance
// is re-scanned from zero over every axis offset, the changed axis taking its
// new offset.
struct Chebyshev {
  static constexpr bool kPeriodic = true;
  static constexpr bool kAdditive = false;
  static constexpr bool kPacked = false;
  template <typename A> __device__ __forceinline__ static A dist1(A a, A b) {
    return abs_val(sub_rn(a, b));
  }
  template <typename A> __device__ __forceinline__ static A combine(A acc, A comp) {
    return comp > acc ? comp : acc;
  }
  template <typename A, int K>
  __device__ __forceinline__ static A rect_k(A, const A (&off)[K], int dim, A new_off) {
    A acc = A(0);
#pragma unroll
    for (int d = 0; d < K; ++d) acc = combine(acc, d == dim ? new_off : off[d]);
    return acc;
  }
};

// ---------------------------------------------------------------------------
// Tree view and the VecOfArenas tile addressing (leaf_view/mod.rs:19-41, 491-505)
// ---------------------------------------------------------------------------
template <typename A>
struct TreeView {
  const A* __restrict__ stems;
  const uint8_t* __restrict__ arena;
  const uint2* __restrict__ extents;  // (byte offset / 8, len)
  int max_stem_level;
  uint32_t leaf_count;
  uint64_t size;
  uint64_t stem_count;
  uint32_t bh;  // 0: Eytzinger stem order; 3 or 4: Donnelly<bh>
  // OwnedStemLeafResolution::Mapped (stem_leaf_resolution.rs:53-66): the leaf
  // of each terminal stem index from map_min on (0xffffffff: not terminal),
  // or null for arithmetic resolution
  const uint32_t* __restrict__ leaf_map;
  uint64_t map_min;
  uint32_t map_len;
};

// resolve_terminal_stem (orchestrator/mod.rs:183-192) for Mapped trees: the
// leaf `stem` maps to, if it is a terminal stem.
template <typename A>
__device__ __forceinline__ bool terminal_leaf(const TreeView<A>& tv, uint32_t stem,
                                              uint32_t& leaf) {
  if (!tv.leaf_map || stem < tv.map_min || uint64_t(stem) - tv.map_min >= tv.map_len) return false;
  const uint32_t l = __ldg(tv.leaf_map + (stem - tv.map_min));
  if (l == 0xffffffffu) return false;
  leaf = l;
  return true;
}

// The two children of a stem at level `level` in the tree's stem order:
// Eytzinger 2i and 2i + 1, Donnelly<bh> as donnelly_children.
template <typename A>
__device__ __forceinline__ void stem_children(const TreeView<A>& tv, uint32_t stem, int level,
                                              uint32_t& l, uint32_t& r);

// Children of a Donnelly<bh> stem (stem_strategy/donnelly/core.rs:400-428):
// inside a minor triangle of bh levels the children of heap slot m of the
// line are slots 2m + 1 and 2m + 2; from the bottom row (minor == bh - 1) they
// are the roots of lines (base + 1 + 2(m - minor - 1) + side) << bh.
__device__ __forceinline__ void donnelly_children(uint32_t stem, uint32_t minor, uint32_t bh,
                                                  uint32_t& left, uint32_t& right) {
  const uint32_t mask = (1u << bh) - 1u;
  const uint32_t min_idx = stem & mask;
  const uint32_t base = (stem & ~mask) + 1u;
  if (minor + 1u == bh) {
    left = (base + ((min_idx - minor - 1u) << 1)) << bh;
    right = left + (1u << bh);
  } else {
    left = base + (min_idx << 1);
    right = left + 1u;
  }
}

// Leaf encoding on the device.  The reference stores a leaf as tiles of 32,
// then 8, 4, 2, 1 points, each tile its K coordinate columns then its items
// (leaf_strategy/vec_of_arenas.rs:292-323).  3-D leaves are held on the
// device instead as one row per point, in the same point order:
//  * f32: 16 bytes, (x, y, z, item bits).  A tile also spends 3 x 4 + 4
//    bytes per point, so every leaf keeps its size and its offset;
//  * f64: 32 bytes, (x, y, z, item bits, 4 zero bytes), against 28 in a tile,
//    so the device arena has offsets of its own (leaf l at 32 x the points
//    before it) and keeps the reference's extents beside them for read-back.
// A point is then one or two aligned 16-byte loads instead of a tile decode
// and four loads.  The arena is converted on upload and back on read-back;
// other shapes keep the tiles.
template <typename A, int K>
struct RowLeaves : std::integral_constant<bool, K == 3> {};
template <typename A>
constexpr uint32_t row_bytes() { return sizeof(A) == 4 ? 16u : 32u; }

// Point p of a leaf held as rows.
template <typename A, int K>
__device__ __forceinline__ void load_row(const uint8_t* __restrict__ leaf, uint32_t p,
                                         A (&c)[K], uint32_t& item) {
  if constexpr (sizeof(A) == 4) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(leaf) + p);
    c[0] = v.x;
    c[1] = v.y;
    c[2] = v.z;
    item = __float_as_uint(v.w);
  } else {
    const double2* r = reinterpret_cast<const double2*>(leaf) + 2 * size_t(p);
    const double2 a = __ldg(r), b = __ldg(r + 1);
    c[0] = a.x;
    c[1] = a.y;
    c[2] = b.x;
    item = uint32_t(__double_as_longlong(b.y));
  }
}

// Byte offset inside the leaf, tile width and index in tile of point p of a
// leaf of `len` points laid out as tiles of 32, then 8, then 4, 2, 1.
template <typename A, int K>
__host__ __device__ __forceinline__ void tile_slot_cols(uint32_t len, uint32_t p, uint32_t& off,
                                                        uint32_t& w, uint32_t& i) {
  constexpr uint32_t per = K * sizeof(A) + sizeof(uint32_t);
  const uint32_t n32 = len >> 5;
  if (p < (n32 << 5)) {
    w = 32; i = p & 31; off = (p >> 5) * (32 * per);
    return;
  }
  uint32_t base = n32 * (32 * per);
  const uint32_t r = len & 31;
  uint32_t pp = p - (n32 << 5);
  const uint32_t n8 = r >> 3;
  if (pp < (n8 << 3)) {
    w = 8; i = pp & 7; off = base + (pp >> 3) * (8 * per);
    return;
  }
  base += n8 * (8 * per);
  pp -= n8 << 3;
  const uint32_t r7 = r & 7;
  if (r7 & 4) {
    if (pp < 4) { w = 4; i = pp; off = base; return; }
    base += 4 * per; pp -= 4;
  }
  if (r7 & 2) {
    if (pp < 2) { w = 2; i = pp; off = base; return; }
    base += 2 * per; pp -= 2;
  }
  w = 1; i = 0; off = base;
}

// The slot of point p in the device encoding: a row is a tile of width 1.
template <typename A, int K>
__device__ __forceinline__ void tile_slot(uint32_t len, uint32_t p, uint32_t& off, uint32_t& w,
                                          uint32_t& i) {
  if constexpr (RowLeaves<A, K>::value) {
    off = p * row_bytes<A>();
    w = 1;
    i = 0;
  } else {
    tile_slot_cols<A, K>(len, p, off, w, i);
  }
}

template <typename A, int K>
__device__ __forceinline__ void load_point(const uint8_t* __restrict__ leaf, uint32_t len,
                                           uint32_t p, A (&c)[K], uint32_t& item) {
  if constexpr (RowLeaves<A, K>::value) {
    load_row<A, K>(leaf, p, c, item);
    return;
  }
  uint32_t off, w, i;
  tile_slot<A, K>(len, p, off, w, i);
  const A* col = reinterpret_cast<const A*>(leaf + off);
#pragma unroll
  for (int d = 0; d < K; ++d) c[d] = __ldg(col + d * w + i);
  item = __ldg(reinterpret_cast<const uint32_t*>(leaf + off + K * w * sizeof(A)) + i);
}

// acc = ((0 + dist1(c0, q0)) + dist1(c1, q1)) + ...   (combine_component order).
// Every dist1 is +0 or more (a square, or fabs), so the leading 0 + dist1 is
// exact and is left out.
template <typename M, typename A, int K>
__device__ __forceinline__ A point_dist(const A (&c)[K], const A (&q)[K]) {
  if constexpr (M::kAdditive) {
    A acc = M::template dist1<A>(c[0], q[0]);
#pragma unroll
    for (int d = 1; d < K; ++d) acc = M::combine(acc, M::template dist1<A>(c[d], q[d]));
    return acc;
  } else {
    // from zero: the first component is combined like the others
    A acc = A(0);
#pragma unroll
    for (int d = 0; d < K; ++d) acc = M::combine(acc, M::template dist1<A>(c[d], q[d]));
    return acc;
  }
}

// Packed pairs of f32 (sm_100 f32x2 arithmetic): each half of a packed sub or
// mul rounds exactly like scalar __fsub_rn / __fmul_rn.  Only sub and mul are
// used packed: the sums stay scalar __fadd_rn in the reference's order (a
// packed multiply followed by a packed add did not reproduce the scalar
// rounding when measured on B200).
struct F2 {
  unsigned long long v;
};
__device__ __forceinline__ F2 f2_pack(float a, float b) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(F2 x, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x.v));
}
__device__ __forceinline__ F2 f2_sub(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 f2_mul(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 f2_abs(F2 a) {  // fabsf on both halves: clear the sign bits
  F2 r;
  r.v = a.v & 0x7fffffff7fffffffull;
  return r;
}

// Largest value below x (x >= 0 or +inf): "d < x" is "d <= below(x)" for
// every non-negative, non-NaN d.
__device__ __forceinline__ float below(float x) {
  return x > 0.f ? __int_as_float(__float_as_int(x) - 1) : -__int_as_float(1);
}
__device__ __forceinline__ double below(double x) {
  return x > 0.0 ? __longlong_as_double(__double_as_longlong(x) - 1)
                 : -__longlong_as_double(1ll);
}

// Point-to-query distance of the Cartesian families.
template <typename A, int K, typename M>
struct CartesianDist {
  __device__ __forceinline__ A operator()(const A (&c)[K], const A (&q)[K]) const {
    return point_dist<M, A, K>(c, q);
  }
};

// Minimum-image distance of the periodic leaf scan (periodic.rs:272-284,
// 357-400): per axis delta = |q - c|, replaced by L - delta when smaller, then
// combine_component(acc, dist1(delta, 0)) from zero.
template <typename A, int K, typename M>
struct PeriodicDist {
  A box[K];
  __device__ __forceinline__ A operator()(const A (&c)[K], const A (&q)[K]) const {
    A acc = A(0);
#pragma unroll
    for (int d = 0; d < K; ++d) {
      const A delta = abs_val(sub_rn(q[d], c[d]));
      const A wrapped = sub_rn(box[d], delta);
      const A m = wrapped < delta ? wrapped : delta;
      acc = M::combine(acc, M::template dist1<A>(m, A(0)));
    }
    return acc;
  }
};


// ---------------------------------------------------------------------------
// The arithmetic traversal, one warp per query.
// Policy interface:
//   A max_dist() const;                       QueryContext::max_dist
//   static constexpr bool kPruneOnEqual;      QueryContext::prune_on_equal_max_dist
//   bool unbounded_start() const;             QueryContext::initial_bound_is_unbounded
//   uint32_t leaf(const TreeView<A>&, uint32_t leaf_idx, const A (&q)[K], int lane);
//     scans one leaf and returns its length.
// ---------------------------------------------------------------------------
// Per-query traversal counters (the counters of test_utils/exact_query_stats.rs:23-60):
// stem visits, leaf visits, points scanned.
struct TravStats {
  uint32_t stems = 0, leaves = 0, points = 0;
};

template <typename A, int K, typename M, typename P>
__device__ __forceinline__ void warp_arith_query(const TreeView<A>& tv, const A (&q)[K], P& pol,
                                                 int lane, TravStats& st) {
  if (tv.size == 0) return;
  const A INF = inf_of<A>();
  const int msl = tv.max_stem_level;
  A off[K];
#pragma unroll
  for (int d = 0; d < K; ++d) off[d] = A(0);
  uint32_t stem_idx = 1;
  int level = 0;
  int dim = 0;
  A rd = A(0);
  uint32_t has_far = 0;             // bit L: a far frame is pending for level L
  A s_old = A(0), s_far = A(0), s_rd = A(0);  // this lane's level-`lane` records

  // arithmetic_descend_to_leaf (orchestrator/mod.rs:520-603)
  auto descend = [&](bool check_bound) -> uint32_t {
    while (level <= msl) {
      ++st.stems;
      const A pivot = __ldg(tv.stems + stem_idx);
      const A oo = sel(off, dim);
      const uint32_t bit = 1u << level;
      if (pivot < INF) {
        const A qd = sel(q, dim);
        const bool is_right = qd >= pivot;
        const A new_off = abs_val(sub_rn(qd, pivot));
        const A rd_far = M::template rect_k<A, K>(rd, off, dim, new_off);
        const bool cand = !check_bound || !(rd_far > pol.max_dist());
        if (lane == level) { s_old = oo; s_far = new_off; s_rd = rd_far; }
        has_far = cand ? (has_far | bit) : (has_far & ~bit);
        stem_idx = stem_idx * 2u + (is_right ? 1u : 0u);
      } else {
        if (lane == level) s_old = oo;
        has_far &= ~bit;
        stem_idx = stem_idx * 2u;
      }
      ++level;
      dim = (dim + 1 == K) ? 0 : dim + 1;
    }
    return stem_idx & ~(1u << level);  // Eytzinger leaf_idx (eytzinger/mod.rs:115-118)
  };

  st.points += pol.leaf(tv, descend(!pol.unbounded_start()), q, lane);
  ++st.leaves;

  // continuation loop (orchestrator/mod.rs:450-515)
  int cur = level;  // stem_idx is the path node at level `cur`
  for (;;) {
    bool resumed = false;
    while (cur > 0) {
      const int L = cur - 1;
      const int d = dim == 0 ? K - 1 : dim - 1;
      dim = d;
      const A old = shfl(s_old, L);
      put(off, d, old);
      const uint32_t bit = 1u << L;
      if (has_far & bit) {
        has_far &= ~bit;
        const A frd = shfl(s_rd, L);
        const A md = pol.max_dist();
        const bool prune = frd > md || (P::kPruneOnEqual && frd == md);
        if (!prune) {
          put(off, d, shfl(s_far, L));
          rd = frd;
          stem_idx ^= 1u;  // the sibling at level L + 1
          level = cur;
          dim = d + 1 == K ? 0 : d + 1;
          st.points += pol.leaf(tv, descend(true), q, lane);
          ++st.leaves;
          cur = level;
          resumed = true;
          break;
        }
      }
      stem_idx >>= 1;
      cur = L;
    }
    if (!resumed) break;
  }
}

// Straight descent for approx (traits/stem_strategy.rs:182-200).
template <typename A>
__device__ __forceinline__ void stem_children(const TreeView<A>& tv, uint32_t stem, int level,
                                              uint32_t& l, uint32_t& r) {
  if (tv.bh) {
    donnelly_children(stem, uint32_t(level) % tv.bh, tv.bh, l, r);
  } else {
    l = stem * 2u;
    r = l + 1u;
  }
}

template <typename A, int K>
__device__ __forceinline__ uint32_t straight_leaf(const TreeView<A>& tv, const A (&q)[K]) {
  if (tv.leaf_map) {
    // get_leaf_idx_mapped (orchestrator/mod.rs:160-178): a terminal stem ends
    // the descent; past max_stem_level the stem maps to its leaf
    uint32_t stem = tv.bh ? 0u : 1u, leaf = 0;
    int dim = 0;
    for (int level = 0; level <= tv.max_stem_level; ++level) {
      if (terminal_leaf(tv, stem, leaf)) return leaf;
      const A pivot = stem < tv.stem_count ? __ldg(tv.stems + stem) : inf_of<A>();
      uint32_t l, r;
      stem_children(tv, stem, level, l, r);
      stem = sel(q, dim) >= pivot ? r : l;
      dim = dim + 1 == K ? 0 : dim + 1;
    }
    terminal_leaf(tv, stem, leaf);  // every terminal is mapped (checked at upload)
    return leaf;
  }
  if (tv.bh) {
    // StemStrategy::get_leaf_idx over Donnelly stems (traits/stem_strategy.rs:
    // 182-200): the leaf index accumulates the path bits.
    uint32_t stem = 0, minor = 0, leaf = 0;
    int dim = 0;
    for (int level = 0; level <= tv.max_stem_level; ++level) {
      const A pivot = stem < tv.stem_count ? __ldg(tv.stems + stem) : inf_of<A>();
      const bool r = sel(q, dim) >= pivot;
      uint32_t l, rr;
      donnelly_children(stem, minor, tv.bh, l, rr);
      stem = r ? rr : l;
      minor = minor + 1u == tv.bh ? 0u : minor + 1u;
      leaf = (leaf << 1) | (r ? 1u : 0u);
      dim = dim + 1 == K ? 0 : dim + 1;
    }
    return leaf;
  }
  uint32_t stem_idx = 1;
  int level = 0, dim = 0;
  while (level <= tv.max_stem_level) {
    const A pivot = __ldg(tv.stems + stem_idx);
    stem_idx = stem_idx * 2u + (sel(q, dim) >= pivot ? 1u : 0u);
    ++level;
    dim = dim + 1 == K ? 0 : dim + 1;
  }
  return stem_idx & ~(1u << level);
}

// ---------------------------------------------------------------------------
// Leaf scans
// ---------------------------------------------------------------------------

// nearest_one leaf kernel (leaf_view_chunked/nearest_one/fallback.rs:69-104):
// sequential `if dist < best` over tile order == first minimum of the leaf
// when it beats the incoming best.  Lanes take points lane, lane+32, ...
template <typename A, int K, typename M>
__device__ __forceinline__ uint32_t scan_nearest_one(const TreeView<A>& tv, uint32_t leaf,
                                                 const A (&q)[K], int lane, A& best,
                                                 uint32_t& best_item) {
  const uint2 ex = __ldg(tv.extents + leaf);
  const uint8_t* base = tv.arena + size_t(ex.x) * 8;
  const uint32_t len = ex.y;
  const A INF = inf_of<A>();
  for (uint32_t b = 0; b < len; b += 32) {
    const uint32_t p = b + lane;
    A dd = INF;
    uint32_t it = 0;
    if (p < len) {
      A c[K];
      load_point<A, K>(base, len, p, c, it);
      dd = point_dist<M, A, K>(c, q);
    }
    A m = dd;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const A other = __shfl_xor_sync(FULL, m, o);
      m = other < m ? other : m;
    }
    if (m < best) {
      const uint32_t hit = __ballot_sync(FULL, p < len && dd == m);
      const int src = __ffs(hit) - 1;
      best = m;
      best_item = shfl(it, src);
    }
  }
  return len;
}

// NearestOne policy (kd_tree/query/nearest_one.rs:321-352)
template <typename A, int K, typename M>
struct NearestOnePolicy {
  static constexpr bool kPruneOnEqual = true;
  A best;
  uint32_t item;
  __device__ NearestOnePolicy() : best(inf_of<A>()), item(0) {}
  __device__ __forceinline__ A max_dist() const { return best; }
  __device__ __forceinline__ bool unbounded_start() const { return true; }
  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint32_t l, const A (&q)[K],
                                           int lane) {
    return scan_nearest_one<A, K, M>(tv, l, q, lane, best, item);
  }
};

// Top-k list in lanes 0..k-1 sorted by (distance, arrival): the
// ThresholdVecResultCollection of result_collection.rs:136-215 with a stable
// fill sort.  Pruning bound = min(k-th distance once full, radius)
// (nearest_n_within.rs:461-468); leaf filter `<=` or `<` against the bound at
// leaf entry (leaf_view_chunked/nearest_n_within/fallback.rs:37-95).
template <typename A, int K, typename M, bool kExclusive, typename PD = CartesianDist<A, K, M>>
struct NearestNPolicy {
  static constexpr bool kPruneOnEqual = kExclusive;
  PD dist;
  A ld;           // lane j: j-th distance
  uint32_t li;    // lane j: j-th item
  uint32_t lseq;  // lane j: arrival number of the j-th entry
  int n;          // entries held (uniform)
  int k;
  A radius;
  A kth;          // ld of lane k-1 once full (uniform)
  uint32_t seq;   // arrivals so far (uniform)
  __device__ NearestNPolicy(int k_, A r, PD pd = PD())
      : dist(pd), ld(inf_of<A>()), li(0xffffffffu), lseq(0), n(0), k(k_), radius(r),
        kth(inf_of<A>()), seq(0) {}
  __device__ __forceinline__ A max_dist() const {
    return (n == k && kth < radius) ? kth : radius;
  }
  __device__ __forceinline__ bool unbounded_start() const { return radius == inf_of<A>(); }

  __device__ __forceinline__ void insert(A cd, uint32_t ci, int lane) {
    const uint32_t le = __ballot_sync(FULL, lane < n && !(ld > cd));
    const int pos = __popc(le);
    const A up_d = shfl_up(ld, 1);
    const uint32_t up_i = shfl_up(li, 1);
    const uint32_t up_s = shfl_up(lseq, 1);
    if (lane > pos) { ld = up_d; li = up_i; lseq = up_s; }
    if (lane == pos) { ld = cd; li = ci; lseq = seq; }
    ++seq;
    if (n < k) ++n;
    kth = shfl(ld, k - 1);
  }

  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint32_t l, const A (&q)[K],
                                           int lane) {
    const uint2 ex = __ldg(tv.extents + l);
    const uint8_t* base = tv.arena + size_t(ex.x) * 8;
    const uint32_t len = ex.y;
    const A bound = max_dist();
    for (uint32_t b = 0; b < len; b += 32) {
      const uint32_t p = b + lane;
      A dd = inf_of<A>();
      uint32_t it = 0;
      bool pass = false;
      if (p < len) {
        A c[K];
        load_point<A, K>(base, len, p, c, it);
        dd = dist(c, q);
        pass = kExclusive ? (dd < bound) : (dd <= bound);
      }
      uint32_t mask = __ballot_sync(FULL, pass);
      if (n == k) mask &= __ballot_sync(FULL, dd < kth);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const A cd = shfl(dd, src);
        const uint32_t ci = shfl(it, src);
        insert(cd, ci, lane);
        if (n == k) mask &= __ballot_sync(FULL, dd < kth);
      }
    }
    return len;
  }

  // Sorted output; `arrival_order` reproduces ThresholdVec::into_vec when the
  // list never filled (arrival order), otherwise the sorted list.
  __device__ __forceinline__ void write(uint64_t qi, A* __restrict__ out_d,
                                        uint32_t* __restrict__ out_i,
                                        uint32_t* __restrict__ out_c, bool arrival_order,
                                        int lane) const {
    int slot = lane;
    if (arrival_order && n < k) {
      // rank of this entry by arrival among the n held entries
      int rank = 0;
      for (int j = 0; j < n; ++j) {
        const uint32_t sj = shfl(lseq, j);
        rank += (sj < lseq) ? 1 : 0;
      }
      slot = rank;
    }
    if (lane < k) {
      const bool valid = lane < n;
      const size_t o = size_t(qi) * k + (valid ? slot : lane);
      out_d[o] = valid ? ld : inf_of<A>();
      out_i[o] = valid ? li : 0xffffffffu;
    }
    if (lane == 0 && out_c) out_c[qi] = uint32_t(n);
  }
};

// nearest_n for 32 < k <= kMaxBigK, one query per warp: the collector of
// NearestNPolicy (ThresholdVec, result_collection.rs:136-215: the k smallest
// by (distance, arrival)), with the list in this warp's shared-memory region
// instead of one entry per lane: distances, items and arrival numbers, kept
// sorted.  An insertion finds its place with one ballot per 32 entries and
// moves the entries above it up by one, 32 at a time from the top.
template <typename A, int K, typename M, bool kExclusive,
          typename PD = CartesianDist<A, K, M>>
struct NearestNBigPolicy {
  static constexpr bool kPruneOnEqual = kExclusive;
  PD dist;
  A* __restrict__ ld;
  uint32_t* __restrict__ li;
  uint32_t* __restrict__ ls;  // arrival number of each entry
  int n, k;
  A radius, kth;
  uint32_t seq;
  __device__ NearestNBigPolicy(A* d, uint32_t* i, uint32_t* s, int k_, A r, PD pd = PD())
      : dist(pd), ld(d), li(i), ls(s), n(0), k(k_), radius(r), kth(inf_of<A>()), seq(0) {}
  __device__ __forceinline__ A max_dist() const {
    return (n == k && kth < radius) ? kth : radius;
  }
  __device__ __forceinline__ bool unbounded_start() const { return radius == inf_of<A>(); }

  __device__ __forceinline__ void insert(A cd, uint32_t ci, int lane) {
    int pos = 0;  // entries not above cd: the new one goes after its equals
    for (int c0 = 0; c0 < n; c0 += 32) {
      const int j = c0 + lane;
      pos += __popc(__ballot_sync(FULL, j < n && !(ld[j] > cd)));
    }
    // entries pos..last move to pos+1..last+1; a full list drops its last
    const int last = n < k ? n - 1 : k - 2;
    if (last >= pos) {
      for (int c0 = last & ~31; c0 >= (pos & ~31); c0 -= 32) {
        const int j = c0 + lane;
        const bool mv = j >= pos && j <= last;
        A d = A(0);
        uint32_t it = 0, sq = 0;
        if (mv) {
          d = ld[j];
          it = li[j];
          sq = ls[j];
        }
        __syncwarp();
        if (mv) {
          ld[j + 1] = d;
          li[j + 1] = it;
          ls[j + 1] = sq;
        }
        __syncwarp();
      }
    }
    if (lane == 0) {
      ld[pos] = cd;
      li[pos] = ci;
      ls[pos] = seq;
    }
    __syncwarp();
    ++seq;
    if (n < k) ++n;
    if (n == k) kth = ld[k - 1];
  }

  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint32_t l, const A (&q)[K],
                                           int lane) {
    const uint2 ex = __ldg(tv.extents + l);
    const uint8_t* base = tv.arena + size_t(ex.x) * 8;
    const uint32_t len = ex.y;
    const A bound = max_dist();
    for (uint32_t b = 0; b < len; b += 32) {
      const uint32_t p = b + lane;
      A dd = inf_of<A>();
      uint32_t it = 0;
      bool pass = false;
      if (p < len) {
        A c[K];
        load_point<A, K>(base, len, p, c, it);
        dd = dist(c, q);
        pass = kExclusive ? (dd < bound) : (dd <= bound);
      }
      uint32_t mask = __ballot_sync(FULL, pass);
      if (n == k) mask &= __ballot_sync(FULL, dd < kth);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        insert(shfl(dd, src), shfl(it, src), lane);
        if (n == k) mask &= __ballot_sync(FULL, dd < kth);
      }
    }
    return len;
  }

  // Sorted rows; with `arrival_order` a list that never filled goes out in
  // arrival order (nothing was evicted, so its arrival numbers are 0..n-1).
  __device__ __forceinline__ void write(uint64_t qi, A* __restrict__ out_d,
                                        uint32_t* __restrict__ out_i,
                                        uint32_t* __restrict__ out_c, bool arrival_order,
                                        int lane) const {
    for (int j = lane; j < k; j += 32) {
      const bool valid = j < n;
      const int slot = (valid && arrival_order && n < k) ? int(ls[j]) : j;
      const size_t o = size_t(qi) * k + slot;
      out_d[o] = valid ? ld[j] : inf_of<A>();
      out_i[o] = valid ? li[j] : 0xffffffffu;
    }
    if (lane == 0 && out_c) out_c[qi] = uint32_t(n);
  }
};

// best_n_within: n smallest items among hits, ties by arrival
// (kd_tree/query/best_n_within.rs:88-196, ctx :281-306; leaf filter
// leaf_view_chunked/best_n_within/fallback.rs:40-104; heap replace-if-smaller
// result_collection.rs:481-501; order by item best_query_result_item.rs:27-31).
template <typename A, int K, typename M, bool kExclusive>
struct BestNPolicy {
  static constexpr bool kPruneOnEqual = kExclusive;
  A ld;
  uint32_t li;
  int n;
  int k;
  A radius;
  __device__ BestNPolicy(int k_, A r) : ld(inf_of<A>()), li(0xffffffffu), n(0), k(k_), radius(r) {}
  __device__ __forceinline__ A max_dist() const { return radius; }
  __device__ __forceinline__ bool unbounded_start() const { return false; }

  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint32_t l, const A (&q)[K],
                                           int lane) {
    const uint2 ex = __ldg(tv.extents + l);
    const uint8_t* base = tv.arena + size_t(ex.x) * 8;
    const uint32_t len = ex.y;
    const bool full_at_entry = n == k;
    const uint32_t thr_item = shfl(li, k - 1);
    for (uint32_t b = 0; b < len; b += 32) {
      const uint32_t p = b + lane;
      A dd = inf_of<A>();
      uint32_t it = 0;
      bool pass = false;
      if (p < len) {
        A c[K];
        load_point<A, K>(base, len, p, c, it);
        dd = point_dist<M, A, K>(c, q);
        pass = kExclusive ? (dd < radius) : (dd <= radius);
        if (full_at_entry && it >= thr_item) pass = false;
      }
      uint32_t mask = __ballot_sync(FULL, pass);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const A cd = shfl(dd, src);
        const uint32_t ci = shfl(it, src);
        if (n == k) {
          const uint32_t last = shfl(li, k - 1);
          if (!(ci < last)) continue;
        }
        const uint32_t le = __ballot_sync(FULL, lane < n && li <= ci);
        const int pos = __popc(le);
        const A up_d = shfl_up(ld, 1);
        const uint32_t up_i = shfl_up(li, 1);
        if (lane > pos) { ld = up_d; li = up_i; }
        if (lane == pos) { ld = cd; li = ci; }
        if (n < k) ++n;
      }
    }
    return len;
  }

  __device__ __forceinline__ void write(uint64_t qi, A* __restrict__ out_d,
                                        uint32_t* __restrict__ out_i,
                                        uint32_t* __restrict__ out_c, int lane) const {
    if (lane < k) {
      const bool valid = lane < n;
      const size_t o = size_t(qi) * k + lane;
      out_d[o] = valid ? ld : inf_of<A>();
      out_i[o] = valid ? li : 0xffffffffu;
    }
    if (lane == 0 && out_c) out_c[qi] = uint32_t(n);
  }
};

// best_n_within for 32 < n <= kMaxBigK, one query per warp: the collector of
// BestNPolicy (the n smallest items among the hits, by (item, arrival);
// best_n_within.rs:88-196) with the list in this warp's shared-memory region,
// kept sorted by item and shifted 32 entries at a time like NearestNBigPolicy.
template <typename A, int K, typename M, bool kExclusive>
struct BestNBigPolicy {
  static constexpr bool kPruneOnEqual = kExclusive;
  A* __restrict__ ld;
  uint32_t* __restrict__ li;
  int n, k;
  A radius;
  __device__ BestNBigPolicy(A* d, uint32_t* i, uint32_t*, int k_, A r)
      : ld(d), li(i), n(0), k(k_), radius(r) {}
  __device__ __forceinline__ A max_dist() const { return radius; }
  __device__ __forceinline__ bool unbounded_start() const { return false; }

  __device__ __forceinline__ void insert(A cd, uint32_t ci, int lane) {
    int pos = 0;  // entries with an item not above ci: the new one goes after them
    for (int c0 = 0; c0 < n; c0 += 32) {
      const int j = c0 + lane;
      pos += __popc(__ballot_sync(FULL, j < n && li[j] <= ci));
    }
    const int last = n < k ? n - 1 : k - 2;
    if (last >= pos) {
      for (int c0 = last & ~31; c0 >= (pos & ~31); c0 -= 32) {
        const int j = c0 + lane;
        const bool mv = j >= pos && j <= last;
        A d = A(0);
        uint32_t it = 0;
        if (mv) {
          d = ld[j];
          it = li[j];
        }
        __syncwarp();
        if (mv) {
          ld[j + 1] = d;
          li[j + 1] = it;
        }
        __syncwarp();
      }
    }
    if (lane == 0) {
      ld[pos] = cd;
      li[pos] = ci;
    }
    __syncwarp();
    if (n < k) ++n;
  }

  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint32_t l, const A (&q)[K],
                                           int lane) {
    const uint2 ex = __ldg(tv.extents + l);
    const uint8_t* base = tv.arena + size_t(ex.x) * 8;
    const uint32_t len = ex.y;
    const bool full_at_entry = n == k;
    const uint32_t thr_item = full_at_entry ? li[k - 1] : 0u;
    for (uint32_t b = 0; b < len; b += 32) {
      const uint32_t p = b + lane;
      A dd = inf_of<A>();
      uint32_t it = 0;
      bool pass = false;
      if (p < len) {
        A c[K];
        load_point<A, K>(base, len, p, c, it);
        dd = point_dist<M, A, K>(c, q);
        pass = kExclusive ? (dd < radius) : (dd <= radius);
        if (full_at_entry && it >= thr_item) pass = false;
      }
      uint32_t mask = __ballot_sync(FULL, pass);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const A cd = shfl(dd, src);
        const uint32_t ci = shfl(it, src);
        if (n == k && !(ci < li[k - 1])) continue;
        insert(cd, ci, lane);
      }
    }
    return len;
  }

  __device__ __forceinline__ void write(uint64_t qi, A* __restrict__ out_d,
                                        uint32_t* __restrict__ out_i,
                                        uint32_t* __restrict__ out_c, bool, int lane) const {
    for (int j = lane; j < k; j += 32) {
      const bool valid = j < n;
      const size_t o = size_t(qi) * k + j;
      out_d[o] = valid ? ld[j] : inf_of<A>();
      out_i[o] = valid ? li[j] : 0xffffffffu;
    }
    if (lane == 0 && out_c) out_c[qi] = uint32_t(n);
  }
};

// within / within().unsorted(): constant bound r (within.rs:18-41,
// within_unsorted.rs:133-157); counting pass and filling pass.
template <typename A, int K, typename M, bool kExclusive, typename PD = CartesianDist<A, K, M>>
struct WithinCountPolicy {
  static constexpr bool kPruneOnEqual = kExclusive;
  PD dist;
  A radius;
  uint64_t count;
  __device__ WithinCountPolicy(A r, PD pd = PD()) : dist(pd), radius(r), count(0) {}
  __device__ __forceinline__ A max_dist() const { return radius; }
  __device__ __forceinline__ bool unbounded_start() const { return radius == inf_of<A>(); }
  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint32_t l, const A (&q)[K],
                                           int lane) {
    const uint2 ex = __ldg(tv.extents + l);
    const uint8_t* base = tv.arena + size_t(ex.x) * 8;
    const uint32_t len = ex.y;
    for (uint32_t b = 0; b < len; b += 32) {
      const uint32_t p = b + lane;
      bool pass = false;
      if (p < len) {
        A c[K];
        uint32_t it;
        load_point<A, K>(base, len, p, c, it);
        const A dd = dist(c, q);
        pass = kExclusive ? (dd < radius) : (dd <= radius);
      }
      count += __popc(__ballot_sync(FULL, pass));
    }
    return len;
  }
};

template <typename A, int K, typename M, bool kExclusive, typename PD = CartesianDist<A, K, M>>
struct WithinFillPolicy {
  static constexpr bool kPruneOnEqual = kExclusive;
  PD dist;
  A radius;
  uint64_t count;
  uint64_t cap;  // the segment length the counting pass produced
  A* __restrict__ out_d;
  uint32_t* __restrict__ out_i;
  __device__ WithinFillPolicy(A r, uint64_t c, A* d, uint32_t* i, PD pd = PD())
      : dist(pd), radius(r), count(0), cap(c), out_d(d), out_i(i) {}
  __device__ __forceinline__ A max_dist() const { return radius; }
  __device__ __forceinline__ bool unbounded_start() const { return radius == inf_of<A>(); }
  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint32_t l, const A (&q)[K],
                                           int lane) {
    const uint2 ex = __ldg(tv.extents + l);
    const uint8_t* base = tv.arena + size_t(ex.x) * 8;
    const uint32_t len = ex.y;
    for (uint32_t b = 0; b < len; b += 32) {
      const uint32_t p = b + lane;
      bool pass = false;
      A dd = A(0);
      uint32_t it = 0;
      if (p < len) {
        A c[K];
        load_point<A, K>(base, len, p, c, it);
        dd = dist(c, q);
        pass = kExclusive ? (dd < radius) : (dd <= radius);
      }
      const uint32_t m = __ballot_sync(FULL, pass);
      if (pass) {
        const uint64_t o = count + __popc(m & ((1u << lane) - 1u));
        if (o < cap) {  // the same traversal as the counting pass: never false
          out_d[o] = dd;
          out_i[o] = it;
        }
      }
      count += __popc(m);
    }
    return len;
  }
};


// ---------------------------------------------------------------------------
// Periodic boundary conditions (kd_tree/query/periodic.rs)
// ---------------------------------------------------------------------------
template <typename A>
__device__ __forceinline__ A max_ref(A a, A b) { return b > a ? b : a; }

// interval_distance_1d (stem_strategy/donnelly/simd_full/mod.rs:209-216)
template <typename A>
__device__ __forceinline__ A interval_distance(A q, A lo, A hi) {
  return add_rn(max_ref(A(0), sub_rn(lo, q)), max_ref(A(0), sub_rn(q, hi)));
}

// periodic_interval_distance_1d (periodic.rs:286-308)
template <typename A>
__device__ __forceinline__ A periodic_interval_distance(A q, A lo, A hi, A L) {
  A best = interval_distance(q, lo, hi);
  const A minus = interval_distance(q, sub_rn(lo, L), sub_rn(hi, L));
  if (minus < best) best = minus;
  const A plus = interval_distance(q, add_rn(lo, L), add_rn(hi, L));
  if (plus < best) best = plus;
  return best;
}

// periodic_backtracking_query (periodic.rs:455-619), one warp per query.  The
// frame stack holds at most one frame per level (frames are pushed at
// increasing levels and popped LIFO), so the frame whose stem sits on level L
// lives in lane L's registers and `has_frame` bit L marks it; popping takes
// the deepest set bit.
template <typename A, int K, typename M, typename P>
__device__ __forceinline__ void warp_periodic_query(const TreeView<A>& tv, const A (&q)[K],
                                                    const A (&box)[K], P& pol, int lane,
                                                    TravStats& st) {
  if (tv.size == 0) return;
  const A INF = inf_of<A>();
  const int msl = tv.max_stem_level;
  uint32_t stem_idx = 1;
  int level = 0, dim = 0;
  A lower[K], upper[K], off[K];
#pragma unroll
  for (int d = 0; d < K; ++d) { lower[d] = A(0); upper[d] = box[d]; off[d] = A(0); }
  A rd = A(0);
  uint32_t has_frame = 0;
  uint32_t f_stem = 0;
  A f_lo[K], f_hi[K], f_off[K], f_rd = A(0);
#pragma unroll
  for (int d = 0; d < K; ++d) { f_lo[d] = A(0); f_hi[d] = A(0); f_off[d] = A(0); }

  auto pop = [&]() -> bool {
    if (!has_frame) return false;
    const int L = 31 - __clz(has_frame);
    has_frame &= ~(1u << L);
    stem_idx = shfl(f_stem, L);
    rd = shfl(f_rd, L);
#pragma unroll
    for (int d = 0; d < K; ++d) {
      lower[d] = shfl(f_lo[d], L);
      upper[d] = shfl(f_hi[d], L);
      off[d] = shfl(f_off[d], L);
    }
    level = L;
    dim = L % K;
    return true;
  };

  for (;;) {
    bool finished = false;
    for (;;) {
      if (level > msl) {
        st.points += pol.leaf(tv, stem_idx & ~(1u << level), q, lane);
        ++st.leaves;
        break;
      }
      ++st.stems;
      const A pivot = stem_idx < tv.stem_count ? __ldg(tv.stems + stem_idx) : INF;
      if (pivot >= INF) {
        stem_idx *= 2u;
        ++level;
        dim = dim + 1 == K ? 0 : dim + 1;
        continue;
      }
      const A old_lo = sel(lower, dim), old_hi = sel(upper, dim);
      const A qd = sel(q, dim), Ld = sel(box, dim);
      const bool is_right = qd >= pivot;
      const uint32_t near_idx = stem_idx * 2u + (is_right ? 1u : 0u);
      const uint32_t far_idx = stem_idx * 2u + (is_right ? 0u : 1u);
      const A minup = old_hi < pivot ? old_hi : pivot;
      const A maxlo = max_ref(old_lo, pivot);
      const A near_lo = is_right ? maxlo : old_lo;
      const A near_hi = is_right ? old_hi : minup;
      const A far_lo = is_right ? old_lo : maxlo;
      const A far_hi = is_right ? minup : old_hi;
      const A near_off = periodic_interval_distance(qd, near_lo, near_hi, Ld);
      const A far_off = periodic_interval_distance(qd, far_lo, far_hi, Ld);
      const A near_rd = M::template rect_k<A, K>(rd, off, dim, near_off);
      const A far_rd = M::template rect_k<A, K>(rd, off, dim, far_off);
      const A thr = pol.max_dist();
      const bool near_pruned = near_rd > thr || (P::kPruneOnEqual && near_rd == thr);
      const bool far_pruned = far_rd > thr || (P::kPruneOnEqual && far_rd == thr);
      if (!far_pruned) {
        const int FL = level + 1;
        if (lane == FL) {
          f_stem = far_idx;
          f_rd = far_rd;
#pragma unroll
          for (int d = 0; d < K; ++d) {
            f_lo[d] = d == dim ? far_lo : lower[d];
            f_hi[d] = d == dim ? far_hi : upper[d];
            f_off[d] = d == dim ? far_off : off[d];
          }
        }
        has_frame |= 1u << FL;
      }
      if (near_pruned) {
        if (pop()) continue;
        finished = true;
        break;
      }
      put(lower, dim, near_lo);
      put(upper, dim, near_hi);
      put(off, dim, near_off);
      rd = near_rd;
      stem_idx = near_idx;
      ++level;
      dim = dim + 1 == K ? 0 : dim + 1;
    }
    if (finished) return;
    if (!pop()) return;
  }
}

constexpr int pow3(int k) { return k == 0 ? 1 : 3 * pow3(k - 1); }

// periodic_nearest_one_result (periodic.rs:156-214): the home query, then each
// image whose lower bound beats the best so far, in (stable) lower-bound order.
// Image j of the 3^K shifts has shift digit (j / 3^(K-1-a)) % 3 - 1 on axis a,
// which is the generation order of periodic_image_candidates (periodic.rs:45-142).
template <typename A, int K, typename M>
__device__ __forceinline__ void warp_periodic_nearest_one(const TreeView<A>& tv, const A (&q)[K],
                                                          const A (&box)[K], int lane, A& best,
                                                          uint32_t& best_item, TravStats& st) {
  {
    NearestOnePolicy<A, K, M> home;
    warp_arith_query<A, K, M>(tv, q, home, lane, st);
    best = home.best;
    best_item = home.item;
  }
  constexpr int NI = pow3(K);
  constexpr int NC = (NI + 31) / 32;
  A wq[NC][K];
  A lb[NC];
  bool valid[NC];
  int rank[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int j = lane + 32 * c;
    int rem = j;
    bool nonzero = false;
    A acc = A(0);
#pragma unroll
    for (int a = 0; a < K; ++a) {
      int div = 1;
      for (int b = a + 1; b < K; ++b) div *= 3;
      const int digit = (rem / div) % 3;
      const A L = box[a];
      const A w = digit == 0 ? sub_rn(q[a], L) : (digit == 1 ? q[a] : add_rn(q[a], L));
      nonzero |= digit != 1;
      wq[c][a] = w;
      // periodic_image_axis_offset (periodic.rs:29-37)
      const A o = w < A(0) ? abs_val(sub_rn(w, A(0))) : (w > L ? abs_val(sub_rn(w, L)) : A(0));
      acc = M::combine(acc, M::template dist1<A>(o, A(0)));
    }
    lb[c] = acc;
    valid[c] = j < NI && nonzero && acc < best;
  }
  // stable rank by lower bound among the valid images
  int nvalid = 0;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    rank[c] = 0;
    nvalid += __popc(__ballot_sync(FULL, valid[c]));
  }
#pragma unroll
  for (int c2 = 0; c2 < NC; ++c2) {
    for (int l2 = 0; l2 < 32; ++l2) {
      const A olb = shfl(lb[c2], l2);
      const bool ov = __shfl_sync(FULL, valid[c2] ? 1u : 0u, l2) != 0u;
      const int oj = l2 + 32 * c2;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const int j = lane + 32 * c;
        if (ov && (olb < lb[c] || (olb == lb[c] && oj < j))) ++rank[c];
      }
    }
  }
  for (int r = 0; r < nvalid; ++r) {
    A img[K];
#pragma unroll
    for (int a = 0; a < K; ++a) img[a] = q[a];
    A ilb = inf_of<A>();
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const uint32_t m = __ballot_sync(FULL, valid[c] && rank[c] == r);
      if (m) {
        const int src = __ffs(m) - 1;
#pragma unroll
        for (int a = 0; a < K; ++a) img[a] = shfl(wq[c][a], src);
        ilb = shfl(lb[c], src);
      }
    }
    if (!(ilb < best)) continue;
    NearestOnePolicy<A, K, M> pol;
    warp_arith_query<A, K, M>(tv, img, pol, lane, st);
    if (pol.best < best) {
      best = pol.best;
      best_item = pol.item;
    }
  }
}

}  // namespace kgpu
