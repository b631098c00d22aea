// kiddo_oracle.hpp — CPU restatement of kiddo's ImmutableKdTree hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker against which the CUDA
// query engine in kiddo_b200/ is compared. Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline / reference leg may load it. The product never
// links or calls it.
//
// It restates, in plain C++17 compiled with -ffp-contract=off (no FMA), the
// default-feature scalar path of kiddo v6.0.0-alpha.3 for
//   ImmutableKdTree<A, K> = KdTree<A, u32, Eytzinger, VecOfArenas<A,u32,K,32>, K, 32>
// Every function cites the reference file:line it follows (paths relative to
// the kiddo repository root).
//
// Parity pin: the literal known-answer tests of the reference (lib.rs:120-151,
// within.rs:115-141, builder.rs:2346-2373, README periodic example, the
// issue-258 within data) are checked in tests/test_oracle_kat.py, and the
// brute-force rules of tests/kd_tree_fuzz_v6.rs:244-340 are checked by property
// tests. The reference itself (Rust) cannot be built in this environment.
//
// Documented choices where the reference depends on unpinned Rust std
// behaviour (std source is not part of the reference):
//  * Intra-leaf order.  Construction uses select_nth_unstable_by
//    (construction.rs:1108); only the k-th order statistic and, under the
//    adjacency property checked by examples/check-select-nth-unstable.rs, the
//    leaf membership are algorithm independent.  This restatement keeps every
//    partition stable, so a leaf lists its points in ascending source index.
//  * ThresholdVec fill sort (result_collection.rs:175-181) is taken as stable:
//    the collector then holds "the k smallest by (distance, arrival order)".
//  * BinaryHeap collectors (k > 192 sorted / > 24 unsorted cartesian, k > 20
//    periodic) keep the same distance multiset as any heap; ties at equal
//    distance are resolved by arrival order here.
//  * Periodic image candidates are sorted stably by lower bound.
#pragma once

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <utility>
#include <vector>

namespace kiddo_oracle {

constexpr size_t kBucket = 32;                    // B of ImmutableKdTree (lib.rs:269-271)
constexpr size_t kTileWidths[5] = {32, 8, 4, 2, 1};  // leaf_view/mod.rs:19
constexpr size_t kLeafScratchCapacity = 1024;     // leaf_view/mod.rs:18

// leaf_view/mod.rs:22-31
inline size_t leaf_arena_tile_len(size_t remaining) {
  for (size_t w : kTileWidths)
    if (remaining >= w) return w;
  return 1;
}

template <typename A>
inline A inf_value() { return std::numeric_limits<A>::infinity(); }

// ---------------------------------------------------------------------------
// Tree layout (kd_tree/mod.rs:221-241, leaf_strategy/vec_of_arenas.rs:60-69)
// ---------------------------------------------------------------------------
template <typename A, int K>
struct Tree {
  std::vector<A> stems;              // stem order of the strategy, +inf = "no split"
  std::vector<uint8_t> leaf_bytes;   // VecOfArenas arena
  std::vector<uint64_t> extents;     // (byte offset, len) pairs per leaf
  int32_t max_stem_level = -1;
  uint64_t size = 0;
  uint64_t max_leaf_len = 0;
  uint32_t stems_depth = 0;
  int stem_strategy = 0;  // 0 Eytzinger, 1 Donnelly<bh>
  uint32_t bh = 0;        // Donnelly block height
  // OwnedStemLeafResolution::Mapped (stem_leaf_resolution.rs:53-66): stem
  // index -> leaf index for terminal stems (kNoLeaf = None), from
  // min_stem_leaf_idx on.  Arithmetic resolution when `mapped` is false.
  static constexpr uint64_t kNoLeaf = ~uint64_t(0);
  bool mapped = false;
  std::vector<uint64_t> leaf_map;
  uint64_t map_min = 0;

  size_t leaf_count() const { return extents.size() / 2; }
  // is_terminal_stem_idx + resolve_terminal_stem_idx (stem_leaf_resolution.rs:
  // 77-120): the stem maps straight to a leaf (Mapped trees only)
  bool terminal(uint64_t stem, size_t* leaf) const {
    if (!mapped || stem < map_min || stem - map_min >= leaf_map.size()) return false;
    const uint64_t l = leaf_map[stem - map_min];
    if (l == kNoLeaf) return false;
    *leaf = size_t(l);
    return true;
  }
  // the leaf of a walk that passed max_stem_level: the map for Mapped trees
  // (which must hold it: the reference panics otherwise), else the arithmetic
  // index
  size_t resolve(uint64_t stem, size_t arithmetic_leaf) const {
    size_t l = arithmetic_leaf;
    if (mapped && !terminal(stem, &l)) return ~size_t(0);
    return l;
  }
  uint64_t leaf_offset(size_t l) const { return extents[2 * l]; }
  uint64_t leaf_len(size_t l) const { return extents[2 * l + 1]; }

  // LeafArena::for_each_tiled_chunk + point_unaligned / item_unaligned
  // (leaf_view/mod.rs:431-446, 491-505): calls f(coords[K], item) in tile order.
  template <typename F>
  void for_each_point(size_t leaf, F&& f) const {
    const uint8_t* base = leaf_bytes.data() + leaf_offset(leaf);
    size_t remaining = leaf_len(leaf);
    size_t byte_off = 0;
    while (remaining) {
      size_t w = leaf_arena_tile_len(remaining);
      const uint8_t* tile = base + byte_off;
      for (size_t i = 0; i < w; ++i) {
        A c[K];
        for (int d = 0; d < K; ++d)
          std::memcpy(&c[d], tile + (d * w + i) * sizeof(A), sizeof(A));
        uint32_t item;
        std::memcpy(&item, tile + K * w * sizeof(A) + i * sizeof(uint32_t), sizeof(uint32_t));
        f(c, item);
      }
      byte_off += K * w * sizeof(A) + w * sizeof(uint32_t);
      remaining -= w;
    }
  }
};

// VecOfArenas::append_leaf (leaf_strategy/vec_of_arenas.rs:292-323)
template <typename A, int K>
void append_leaf(Tree<A, K>& t, const A* pts, const uint32_t* items, const size_t* idx,
                 size_t len) {
  const size_t align = std::max<size_t>(std::max(alignof(A), alignof(uint32_t)), 8);
  size_t start = (t.leaf_bytes.size() + align - 1) & ~(align - 1);
  t.leaf_bytes.resize(start, 0);
  t.extents.push_back(start);
  t.extents.push_back(len);
  size_t base = 0;
  size_t remaining = len;
  while (remaining) {
    size_t w = leaf_arena_tile_len(remaining);
    for (int d = 0; d < K; ++d)
      for (size_t i = 0; i < w; ++i) {
        A v = pts[idx[base + i] * K + d];
        const uint8_t* p = reinterpret_cast<const uint8_t*>(&v);
        t.leaf_bytes.insert(t.leaf_bytes.end(), p, p + sizeof(A));
      }
    for (size_t i = 0; i < w; ++i) {
      uint32_t it = items[idx[base + i]];
      const uint8_t* p = reinterpret_cast<const uint8_t*>(&it);
      t.leaf_bytes.insert(t.leaf_bytes.end(), p, p + sizeof(uint32_t));
    }
    base += w;
    remaining -= w;
  }
}

// ---------------------------------------------------------------------------
// Stem orderings (traits/stem_strategy.rs): the position of a node in the
// stem array, its level, its split dimension and its leaf-index prefix.
// ---------------------------------------------------------------------------
// Eytzinger (stem_strategy/eytzinger/mod.rs:81-186): root 1, children 2i and
// 2i + 1, dim = level % K.
template <int K>
struct EytzingerCursor {
  uint32_t stem_idx = 1;
  int level = 0;
  int dim() const { return level % K; }
  EytzingerCursor branch() {  // self -> left child, returns the right child
    EytzingerCursor r = *this;
    stem_idx *= 2;
    ++level;
    r.stem_idx = stem_idx + 1;
    r.level = level;
    return r;
  }
  // the arithmetic leaf index: stem_idx without its leading bit
  size_t leaf_idx() const { return size_t(stem_idx & ~(uint32_t(1) << level)); }
  void traverse(bool is_right) {
    stem_idx = stem_idx * 2 + (is_right ? 1u : 0u);
    ++level;
  }
  // self -> near child, returns the far one (traits/stem_strategy.rs:110-118)
  EytzingerCursor branch_relative(bool is_right) {
    EytzingerCursor far = *this;
    far.traverse(!is_right);
    traverse(is_right);
    return far;
  }
};

// DonnellyCore<BH> (stem_strategy/donnelly/core.rs:35-154, 254-290, 400-428):
// stems packed in minor triangles of BH levels, each a 0-based heap inside a
// line of 2^BH slots; the child triangles of a triangle's bottom row start at
// line (line_base + 1 + 2 * col + is_right) << BH, col = min_idx - minor - 1.
// dim advances once per level (wrapping at K); leaf_idx accumulates the path
// bits, which is the arithmetic leaf index of an immutable tree
// (kd_tree/mod.rs:164-178).
template <int K>
struct DonnellyCursor {
  uint32_t bh = 3;
  uint32_t stem_idx = 0;
  int level = 0;
  uint32_t minor = 0;
  uint64_t leaf_idx = 0;
  int dim_ = 0;
  int dim() const { return dim_; }
  uint32_t line_mask() const { return (1u << bh) - 1u; }

  // step_pure (core.rs:254-290)
  void traverse(bool is_right) {
    const uint32_t r = is_right ? 1u : 0u;
    const uint32_t min_idx = stem_idx & line_mask();
    const uint32_t min_col = min_idx - minor - 1u;
    const uint32_t base_no_right = (stem_idx & ~line_mask()) + 1u;
    const uint32_t next_base = (base_no_right + (min_col << 1)) << bh;
    const uint32_t same = base_no_right + r + (min_idx << 1);
    const uint32_t next = next_base + (r << bh);
    const bool inc_major = minor + 1u == bh;
    stem_idx = inc_major ? next : same;
    minor = inc_major ? 0u : minor + 1u;
    advance(is_right);
  }
  // both_children_pure (core.rs:400-428)
  void children(uint32_t& left, uint32_t& right) const {
    const uint32_t min_idx = stem_idx & line_mask();
    const uint32_t min_row = min_idx - minor - 1u;
    const bool inc_major = minor + 1u == bh;
    const uint32_t base_no_right = (stem_idx & ~line_mask()) + 1u;
    const uint32_t same_left = base_no_right + (min_idx << 1);
    const uint32_t next_left = (base_no_right + (min_row << 1)) << bh;
    left = inc_major ? next_left : same_left;
    right = inc_major ? next_left + (1u << bh) : same_left + 1u;
  }
  // branch (core.rs:124-148): self -> left child, returns the right child
  DonnellyCursor branch() {
    uint32_t l, r;
    children(l, r);
    stem_idx = l;
    minor = minor + 1u == bh ? 0u : minor + 1u;
    advance(false);
    DonnellyCursor right = *this;
    right.stem_idx = r;
    right.leaf_idx = leaf_idx | 1u;
    return right;
  }
  // branch_relative (traits/stem_strategy.rs:110-118): self -> near child,
  // returns the far one
  DonnellyCursor branch_relative(bool is_right) {
    DonnellyCursor right = branch();
    if (!is_right) return right;
    DonnellyCursor left = *this;
    *this = right;
    return left;
  }

 private:
  void advance(bool is_right) {
    ++level;
    dim_ = dim_ == K - 1 ? 0 : dim_ + 1;
    leaf_idx = (leaf_idx << 1) | (is_right ? 1u : 0u);
  }
};

// ---------------------------------------------------------------------------
// Construction: soft-bucket bulk build (construction.rs:413-539, 868-968)
// ---------------------------------------------------------------------------
template <typename A, int K>
struct Builder {
  const A* pts;
  const uint32_t* items;
  Tree<A, K>* t;
  std::vector<size_t> tmp;

  A coord(size_t i, int d) const { return pts[i * K + d]; }

  // update_pivot (construction.rs:1089-1175).  Restated through counts:
  // after select_nth the nudge-left loop stops at the first slot of the run
  // equal to v (= count(< v)); when that reaches 0 the sorted nudge-right ends
  // after the run (= count(<= v)) or declares the chunk unsplittable (= len).
  size_t update_pivot(size_t* idx, size_t len, int dim, size_t init_pivot) {
    std::vector<A> vals(len);
    for (size_t i = 0; i < len; ++i) vals[i] = coord(idx[i], dim);
    std::nth_element(vals.begin(), vals.begin() + init_pivot, vals.end());
    const A v = vals[init_pivot];
    size_t lt = 0, le = 0;
    for (size_t i = 0; i < len; ++i) {
      A x = coord(idx[i], dim);
      lt += (x < v);
      le += (x <= v);
    }
    if (lt > 0) return lt;
    if (le >= len) return len;
    return le;
  }

  // Stable partition of idx[0..len) so that the first `pivot` entries are the
  // `pivot` smallest on `dim` (a prefix of the value order, which is exactly
  // {x < v} or {x <= v} for the pivots update_pivot returns).
  void stable_split(size_t* idx, size_t len, int dim, size_t pivot) {
    if (pivot == 0 || pivot >= len) return;
    // threshold value: the pivot-th smallest
    std::vector<A> vals(len);
    for (size_t i = 0; i < len; ++i) vals[i] = coord(idx[i], dim);
    std::nth_element(vals.begin(), vals.begin() + pivot, vals.end());
    const A v = vals[pivot];  // smallest value of the right part
    tmp.resize(len);
    size_t l = 0, r = pivot;
    for (size_t i = 0; i < len; ++i) {
      if (coord(idx[i], dim) < v) tmp[l++] = idx[i];
      else tmp[r++] = idx[i];
    }
    std::copy(tmp.begin(), tmp.begin() + len, idx);
  }

  // populate_recursive_soft (construction.rs:868-968), generic over the stem
  // ordering as the reference is (EytzingerCursor / DonnellyCursor).
  template <typename Cursor>
  void populate(size_t* idx, size_t len, Cursor cur, int max_stem_level, uint64_t leaf_budget) {
    if (leaf_budget == 0) return;
    const int level = cur.level;
    const uint32_t stem_idx = cur.stem_idx;
    if (level > max_stem_level) {
      // write_leaf_from_sort_index (construction.rs:641-670)
      t->max_leaf_len = std::max<uint64_t>(t->max_leaf_len, len);
      append_leaf(*t, pts, items, idx, len);
      return;
    }
    const int dim = cur.dim();
    t->max_stem_level = std::max(t->max_stem_level, level);
    if (stem_idx >= t->stems.size()) t->stems.resize(stem_idx + 1, inf_value<A>());

    uint64_t left_budget, right_budget;
    size_t pivot;
    if (leaf_budget == 1) {
      left_budget = 1;
      right_budget = 0;
      pivot = len;
    } else {
      // soft_left_leaf_budget (construction.rs:673-676): largest power of two < budget
      left_budget = uint64_t(1) << (63 - __builtin_clzll(leaf_budget - 1));
      right_budget = leaf_budget - left_budget;
      // soft_ideal_pivot (construction.rs:679-691)
      if (len == 0) {
        pivot = 0;
      } else {
        unsigned __int128 num = (unsigned __int128)len * left_budget;
        size_t p = (size_t)((num + leaf_budget - 1) / leaf_budget);
        pivot = std::min(std::max<size_t>(p, 1), len);
      }
      if (pivot < len) pivot = update_pivot(idx, len, dim, pivot);
    }
    if (pivot < len) {
      stable_split(idx, len, dim, pivot);
      // stems[stem_index] = axis_at(source[sort_index[pivot]], dim): the
      // smallest coordinate of the right part.
      A m = coord(idx[pivot], dim);
      for (size_t i = pivot; i < len; ++i) m = std::min(m, coord(idx[i], dim));
      t->stems[stem_idx] = m;
    }
    const size_t split = std::min(pivot, len);
    Cursor right = cur.branch();
    populate(idx, split, cur, max_stem_level, left_budget);
    populate(idx + split, len - split, right, max_stem_level, right_budget);
  }
};

// ---------------------------------------------------------------------------
// Construction: hard-bucket bulk build for mutable leaf strategies
// (MutableKdTree = KdTree<A, u32, Eytzinger, VecOfArrays<A, u32, K, 32>, K, 32>,
// lib.rs:274-275; construction.rs:413-539, 695-864, 972-1009, 1039-1085)
// ---------------------------------------------------------------------------
// calc_pivot (construction.rs:1039-1085) for hard buckets: the left part is
// filled up to a multiple of B, at least B where the chunk allows; a split
// that would leave everything on the left (and more than B there) puts
// max(right_capacity, B) on the right instead.
inline size_t hard_calc_pivot(size_t len, size_t right_capacity) {
  auto next_multiple = [](size_t x) { return (x + kBucket - 1) / kBucket * kBucket; };
  const size_t sat = len > right_capacity ? len - right_capacity : 0;
  size_t result = std::min(next_multiple(sat), len);
  if (len > 0) result = std::max(result, std::min(kBucket, len));
  if (result >= len && result > kBucket) {
    const size_t rc = std::max(right_capacity, kBucket);
    const size_t sat2 = len > rc ? len - rc : 0;
    result = std::min(next_multiple(sat2), len);
  }
  return result;
}

template <typename A, int K>
struct HardBuilder {
  Builder<A, K>& b;
  Tree<A, K>& t;
  std::vector<uint64_t> terminals;  // terminal stem index of each leaf, in leaf order
  bool unsplittable = false;

  // populate_recursive_hard (construction.rs:695-864)
  template <typename Cursor>
  void populate(size_t* idx, size_t len, Cursor cur, int max_stem_level, size_t capacity) {
    if (unsplittable || len == 0) return;
    if (len <= kBucket) {
      t.max_leaf_len = std::max<uint64_t>(t.max_leaf_len, len);
      append_leaf(t, b.pts, b.items, idx, len);
      terminals.push_back(cur.stem_idx);
      return;
    }
    const int levels_below = std::max(max_stem_level - cur.level, 0);
    const size_t left_capacity =
        std::min(levels_below >= 60 ? capacity : (size_t(1) << levels_below) * kBucket, capacity);
    const size_t right_capacity = capacity > left_capacity ? capacity - left_capacity : 0;
    const uint32_t stem_index = cur.stem_idx;
    t.max_stem_level = std::max(t.max_stem_level, cur.level);
    if (stem_index >= t.stems.size()) t.stems.resize(stem_index + 1, inf_value<A>());
    const int dim = cur.dim();
    size_t pivot = hard_calc_pivot(len, right_capacity);
    if (pivot < len) {
      pivot = b.update_pivot(idx, len, dim, pivot);
      if (pivot >= len) {  // ConstructionError::UnsplittableBucket (construction.rs:1146-1148)
        unsplittable = true;
        return;
      }
      b.stable_split(idx, len, dim, pivot);
      A m = b.coord(idx[pivot], dim);
      for (size_t i = pivot; i < len; ++i) m = std::min(m, b.coord(idx[i], dim));
      t.stems[stem_index] = m;
    }
    Cursor right = cur.branch();
    populate(idx, pivot, cur, max_stem_level, left_capacity);
    if (len > pivot) populate(idx + pivot, len - pivot, right, max_stem_level, right_capacity);
  }
};

// new_from_source_with for a mutable, hard-bucket leaf strategy: the stem
// tree sized by walking to leaf leaf_node_count - 1 below the root
// (construction.rs:448-469), populate_recursive_hard, then Mapped resolution
// from the terminal stems in leaf order (mapped_stem_leaf_resolution_from_
// terminals, :972-1009); a tree of fewer than two leaves has no stems and maps
// the root stem to its leaf (build_mapped_stem_leaf_resolution,
// traits/leaf_strategy.rs:30-76).  Returns false for an unsplittable bucket.
template <typename A, int K>
bool build_hard(Tree<A, K>& t, const A* pts, const uint32_t* items, size_t n, uint32_t bh = 0) {
  t = Tree<A, K>();
  t.size = n;
  t.stem_strategy = bh ? 1 : 0;
  t.bh = bh;
  t.mapped = true;
  t.map_min = 0;
  const size_t leaf_node_count = (n + kBucket - 1) / kBucket;
  std::vector<size_t> idx(n);
  std::iota(idx.begin(), idx.end(), size_t(0));
  if (leaf_node_count < 2) {
    t.max_stem_level = -1;
    if (n == 0) return true;
    t.max_leaf_len = n;
    append_leaf(t, pts, items, idx.data(), n);
    const uint64_t root = bh ? 0 : 1;
    t.leaf_map.assign(root + 1, Tree<A, K>::kNoLeaf);
    t.leaf_map[root] = 0;
    return true;
  }
  uint32_t depth = 0;
  while ((size_t(1) << depth) < leaf_node_count) ++depth;
  Builder<A, K> b{pts, items, &t, {}};
  HardBuilder<A, K> hb{b, t, {}, false};
  t.max_stem_level = -1;
  auto run = [&](auto root, uint32_t padded_depth) {
    auto walk = root;
    for (int bit = int(padded_depth) - 1; bit >= 1; --bit)
      walk.traverse(((leaf_node_count - 1) >> bit) & 1u);
    const size_t stem_node_count = size_t(walk.stem_idx) + 1;
    t.stems.assign((stem_node_count + 7) / 8 * 8, inf_value<A>());
    hb.populate(idx.data(), n, root, int(padded_depth) - 1, leaf_node_count * kBucket);
  };
  if (!bh) {
    t.stems_depth = depth;
    run(EytzingerCursor<K>{}, depth);
  } else {
    const uint32_t padding = depth % bh ? bh - depth % bh : 0;
    depth += padding;
    t.stems_depth = depth;
    DonnellyCursor<K> root;
    root.bh = bh;
    for (uint32_t i = 0; i < padding; ++i) root.traverse(false);
    run(root, depth);
  }
  if (hb.unsplittable) return false;
  uint64_t max_terminal = 0;
  for (uint64_t s : hb.terminals) max_terminal = std::max(max_terminal, s);
  t.leaf_map.assign(max_terminal + 1, Tree<A, K>::kNoLeaf);
  for (size_t l = 0; l < hb.terminals.size(); ++l) t.leaf_map[hb.terminals[l]] = l;
  return true;
}

// A Mapped tree of irregular depth, as a MutableKdTree holds after leaf
// splits (construction.rs:19-130): from each node, a chunk of at most B
// points becomes a leaf with probability 1/2 (always once it has one point,
// or cannot be split), a larger one is split at its median by the
// reference's pivot rule.  Test data for the Mapped traversal, not a
// restatement of the reference's mutation sequence.
template <typename A, int K>
void build_irregular(Tree<A, K>& t, const A* pts, const uint32_t* items, size_t n,
                     uint64_t seed) {
  t = Tree<A, K>();
  t.size = n;
  t.mapped = true;
  t.max_stem_level = -1;
  std::vector<size_t> idx(n);
  std::iota(idx.begin(), idx.end(), size_t(0));
  Builder<A, K> b{pts, items, &t, {}};
  std::vector<uint64_t> terminals;
  uint64_t rng = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto coin = [&]() {
    rng = rng * 6364136223846793005ull + 1442695040888963407ull;
    return (rng >> 33) & 1u;
  };
  std::function<void(size_t*, size_t, EytzingerCursor<K>)> rec = [&](size_t* ix, size_t len,
                                                                     EytzingerCursor<K> cur) {
    const int dim = cur.dim();
    size_t pivot = len;
    if (len > 1 && cur.level < 30 && (len > kBucket || coin()))
      pivot = b.update_pivot(ix, len, dim, len / 2 ? len / 2 : 1);
    if (pivot >= len || pivot == 0) {
      t.max_leaf_len = std::max<uint64_t>(t.max_leaf_len, len);
      append_leaf(t, pts, items, ix, len);
      terminals.push_back(cur.stem_idx);
      return;
    }
    t.max_stem_level = std::max(t.max_stem_level, cur.level);
    if (cur.stem_idx >= t.stems.size()) t.stems.resize(cur.stem_idx + 1, inf_value<A>());
    b.stable_split(ix, len, dim, pivot);
    A m = b.coord(ix[pivot], dim);
    for (size_t i = pivot; i < len; ++i) m = std::min(m, b.coord(ix[i], dim));
    t.stems[cur.stem_idx] = m;
    EytzingerCursor<K> right = cur.branch();
    rec(ix, pivot, cur);
    rec(ix + pivot, len - pivot, right);
  };
  if (n) rec(idx.data(), n, EytzingerCursor<K>{});
  uint64_t max_terminal = 0;
  for (uint64_t s : terminals) max_terminal = std::max(max_terminal, s);
  t.leaf_map.assign(n ? max_terminal + 1 : 0, Tree<A, K>::kNoLeaf);
  for (size_t l = 0; l < terminals.size(); ++l) t.leaf_map[terminals[l]] = l;
}

// KdTree::new_from_entries / new_from_slice -> new_from_source_with
// (construction.rs:278-303, 403-409, 413-539, 540-589).  bh == 0 builds the
// Eytzinger layout (ImmutableKdTree); bh > 0 builds Donnelly<bh>, whose stem
// tree is padded at the root to a multiple of bh levels (construction.rs:
// 431-446) and sized by walking to the right-most leaf (:448-469).
template <typename A, int K>
Tree<A, K> build(const A* pts, const uint32_t* items, size_t n, uint32_t bh = 0) {
  Tree<A, K> t;
  t.size = n;
  t.stem_strategy = bh ? 1 : 0;
  t.bh = bh;
  const size_t leaf_node_count = (n + kBucket - 1) / kBucket;
  std::vector<size_t> idx(n);
  std::iota(idx.begin(), idx.end(), size_t(0));
  if (leaf_node_count < 2) {
    // new_from_source_no_stems_with: a single leaf, no stems.
    if (n == 0) return t;
    t.max_stem_level = -1;
    t.max_leaf_len = n;
    append_leaf(t, pts, items, idx.data(), n);
    return t;
  }
  // stems_depth = log2(next_power_of_two(leaf_node_count))
  uint32_t depth = 0;
  while ((size_t(1) << depth) < leaf_node_count) ++depth;
  Builder<A, K> b{pts, items, &t, {}};
  t.max_stem_level = -1;
  if (!bh) {
    t.stems_depth = depth;
    const uint64_t budget = uint64_t(1) << depth;
    // stem_node_count: index of the right-most represented leaf + 1, padded to 8.
    const size_t stem_node_count = (size_t(1) << (depth + 1));
    const size_t padded = (stem_node_count + 7) / 8 * 8;
    t.stems.assign(padded, inf_value<A>());
    b.populate(idx.data(), n, EytzingerCursor<K>{}, int(depth) - 1, budget);
    return t;
  }
  uint32_t padding = depth % bh ? bh - depth % bh : 0;
  depth += padding;
  t.stems_depth = depth;
  DonnellyCursor<K> root;
  root.bh = bh;
  for (uint32_t i = 0; i < padding; ++i) root.traverse(false);
  const uint64_t budget = uint64_t(1) << depth;
  DonnellyCursor<K> right_most = root;
  for (int bit = int(depth) - 1; bit >= 0; --bit) right_most.traverse(((budget - 1) >> bit) & 1u);
  const size_t stem_node_count = size_t(right_most.stem_idx) + 1;
  t.stems.assign((stem_node_count + 7) / 8 * 8, inf_value<A>());
  b.populate(idx.data(), n, root, int(depth) - 1, budget);
  return t;
}

// ---------------------------------------------------------------------------
// Distance metrics (dist/distance_metric_core.rs:12-105,
// dist/squared_euclidean/mod.rs:21-40, dist/manhattan/mod.rs:21-48,
// traits/axis.rs:82-139)
// ---------------------------------------------------------------------------
// The additive metrics: combine_component is acc += component, and the
// rectangle distance after one axis offset changes is the O(1) update
// (rd - dist1(old, 0)) + dist1(new, 0) (distance_metric_core.rs:86-96).
template <typename Self>
struct Additive {
  static constexpr bool kPeriodic = true;  // restated for periodic queries
  template <typename A> static A combine(A acc, A component) { return acc + component; }
  template <typename A, int K>
  static A rect_k(A rd, const A* off, int dim, A new_off) {
    return Self::rect_after_update(rd, off[dim], new_off);
  }
};
struct SqEuclidean : Additive<SqEuclidean> {
  template <typename A> static A dist1(A a, A b) { A d = a - b; return d * d; }
  template <typename A> static A rect_after_update(A rd, A old_off, A new_off) {
    A new1 = dist1(new_off, A(0));
    A old1 = dist1(old_off, A(0));
    return (rd - old1) + new1;
  }
};
struct Manhattan : Additive<Manhattan> {
  template <typename A> static A dist1(A a, A b) { return std::fabs(a - b); }
  template <typename A> static A rect_after_update(A rd, A old_off, A new_off) {
    return (rd - old_off) + new_off;
  }
};
// Chebyshev / L-infinity (dist/chebyshev/mod.rs:19-59): dist1 = |a - b|
// (Axis::saturating_dist), combine_component keeps the larger value (a
// component that is not greater, NaN included, leaves acc unchanged), and the
// rectangle distance is re-scanned from zero over every axis offset, the
// changed axis taking its new offset.
struct Chebyshev {
  static constexpr bool kPeriodic = true;
  template <typename A> static A dist1(A a, A b) { return std::fabs(a - b); }
  template <typename A> static A combine(A acc, A component) {
    return component > acc ? component : acc;
  }
  template <typename A, int K>
  static A rect_k(A, const A* off, int dim, A new_off) {
    A acc = A(0);
    for (int axis = 0; axis < K; ++axis) acc = combine(acc, axis == dim ? new_off : off[axis]);
    return acc;
  }
};

// Minkowski<P> (dist/minkowski/mod.rs:19-58): dist1 = |a - b|.powi(P), the
// sum of powered differences without the final root.  Rust's powi is LLVM's
// llvm.powi, which is expanded by binary exponentiation (result times the
// running square, low bit first): x^3 = x * (x * x), x^4 = (x * x) * (x * x).
// Restated for P = 3 and 4.
template <int P>
inline double powi_binary(double x) {
  double res = 1.0, cur = x;
  bool have = false;
  for (int e = P; e; e >>= 1) {
    if (e & 1) {
      res = have ? res * cur : cur;
      have = true;
    }
    if (e >> 1) cur = cur * cur;
  }
  return res;
}
template <int P>
inline float powi_binary(float x) {
  float res = 1.f, cur = x;
  bool have = false;
  for (int e = P; e; e >>= 1) {
    if (e & 1) {
      res = have ? res * cur : cur;
      have = true;
    }
    if (e >> 1) cur = cur * cur;
  }
  return res;
}
template <int P>
struct Minkowski : Additive<Minkowski<P>> {
  template <typename A> static A dist1(A a, A b) { return powi_binary<P>(std::fabs(a - b)); }
  template <typename A> static A rect_after_update(A rd, A old_off, A new_off) {
    return (rd - dist1(old_off, A(0))) + dist1(new_off, A(0));
  }
};

// combine_component over dist1(point, query), left to right from zero.
template <typename M, typename A, int K>
inline A point_dist(const A* c, const A* q) {
  A acc = A(0);
  for (int d = 0; d < K; ++d) acc = M::combine(acc, M::template dist1<A>(c[d], q[d]));
  return acc;
}

// ---------------------------------------------------------------------------
// Statistics used for the algorithmic-bytes model (the counters of
// test_utils/exact_query_stats.rs:23-60).
// ---------------------------------------------------------------------------
struct Stats {
  uint64_t stem_visits = 0;
  uint64_t leaf_visits = 0;
  uint64_t points_scanned = 0;
};

// ---------------------------------------------------------------------------
// Arithmetic Eytzinger traversal with continuation stacks
// (kd_tree/orchestrator/mod.rs:388-516 arithmetic_query_with_scratch_impl,
//  :520-603 arithmetic_descend_to_leaf).  The query context supplies
//  max_dist(), initial_bound_is_unbounded(), prune_on_equal()
//  (kd_tree/query_context.rs:6-35).
// ---------------------------------------------------------------------------
template <typename A, int K, typename M, typename Ctx, typename Leaf>
void arithmetic_query(const Tree<A, K>& t, const A* q, Ctx& ctx, Leaf&& process_leaf,
                      Stats* st) {
  if (t.size == 0) return;
  struct Restore { A old_off; bool has_far; };
  struct Far { uint32_t stem_idx; int level; A far_off; A rd; };
  Restore restore_stack[72];
  Far far_stack[72];
  int rs_len = 0, fs_len = 0;

  A off[K];
  for (int d = 0; d < K; ++d) off[d] = A(0);
  uint32_t stem_idx = 1;
  int level = 0;
  A rd = A(0);
  const A INF = inf_value<A>();

  auto descend = [&](bool check_bound) -> size_t {
    while (level <= t.max_stem_level) {
      if (st) st->stem_visits++;
      const int dim = level % K;
      const A pivot = t.stems[stem_idx];
      if (pivot < INF) {
        const A qd = q[dim];
        const bool is_right = qd >= pivot;
        const uint32_t near_idx = stem_idx * 2 + (is_right ? 1u : 0u);
        const uint32_t far_idx = stem_idx * 2 + (is_right ? 0u : 1u);
        const A new_off = std::fabs(qd - pivot);  // Axis::saturating_dist
        const A old_off = off[dim];
        const A rd_far = M::template rect_k<A, K>(rd, off, dim, new_off);
        bool far_is_candidate = true;
        if (check_bound) far_is_candidate = !(rd_far > ctx.max_dist());
        if (far_is_candidate) {
          restore_stack[rs_len++] = {old_off, true};
          far_stack[fs_len++] = {far_idx, level + 1, new_off, rd_far};
        } else {
          restore_stack[rs_len++] = {old_off, false};
        }
        stem_idx = near_idx;
      } else {
        restore_stack[rs_len++] = {off[dim], false};
        stem_idx = stem_idx * 2;
      }
      ++level;
    }
    // Eytzinger leaf_idx: stem_idx & !(1 << level) (eytzinger/mod.rs:115-118)
    return size_t(stem_idx & ~(uint32_t(1) << level));
  };

  auto visit = [&](size_t leaf) {
    if (st) { st->leaf_visits++; st->points_scanned += t.leaf_len(leaf); }
    process_leaf(leaf);
  };

  visit(descend(!ctx.initial_bound_is_unbounded()));
  int dim = level % K;
  for (;;) {
    bool resumed = false;
    while (rs_len > 0) {
      Restore fr = restore_stack[--rs_len];
      const int restore_dim = dim == 0 ? K - 1 : dim - 1;
      off[restore_dim] = fr.old_off;
      dim = restore_dim;
      if (!fr.has_far) continue;
      Far far = far_stack[--fs_len];
      const A md = ctx.max_dist();
      const bool prune = far.rd > md || (ctx.prune_on_equal() && far.rd == md);
      if (prune) continue;
      restore_stack[rs_len++] = {fr.old_off, false};
      off[restore_dim] = far.far_off;
      stem_idx = far.stem_idx;
      level = far.level;
      rd = far.rd;
      visit(descend(true));
      dim = level % K;
      resumed = true;
      break;
    }
    if (!resumed) break;
  }
}

// Scalar backtracking with an explicit stack, the path of every strategy
// whose BLOCK_SIZE != 1 (Donnelly; orchestrator/mod.rs:214-345, 607-669,
// traits/stem_strategy.rs:209-325, query_stack.rs:124-200).  A frame holds
// the far child's stem state, the dimension to restore, the off value to put
// there and the far child's rd.  The prune test is made when a frame is
// popped; on the way down `rd` stays the popped frame's, and the far child is
// pushed when rd_far is not greater than max_dist() as read when the descent
// started.  Only the popped frame's own dimension of `off` is reset, so
// values set under deeper subtrees carry over, as in the reference.
template <int K>
inline size_t cursor_leaf(const EytzingerCursor<K>& c) { return c.leaf_idx(); }
template <int K>
inline size_t cursor_leaf(const DonnellyCursor<K>& c) { return size_t(c.leaf_idx); }

// Over the stem order of cursor C (DonnellyCursor, or EytzingerCursor for a
// Mapped Eytzinger tree), with the Mapped resolution's terminal-stem checks of
// traverse_to_leaf (orchestrator/mod.rs:607-669): a stem that maps to a leaf
// ends the descent there.
template <typename A, int K, typename M, typename C, typename Ctx, typename Leaf>
void scalar_backtracking_query_c(const Tree<A, K>& t, C root, const A* q, Ctx& ctx,
                                 Leaf&& process_leaf, Stats* st) {
  if (t.size == 0) return;
  struct Frame {
    C s;
    int restore_dim;  // -1: the popped state's own dimension
    A old_off;
    A rd;
  };
  std::vector<Frame> stack;
  stack.push_back({root, -1, A(0), A(0)});
  A off[K];
  for (int d = 0; d < K; ++d) off[d] = A(0);
  const A INF = inf_value<A>();
  while (!stack.empty()) {
    Frame f = stack.back();
    stack.pop_back();
    C s = f.s;
    int dim = s.dim();
    const int restore_dim = f.restore_dim < 0 ? dim : f.restore_dim;
    const A md = ctx.max_dist();
    if (f.rd > md || (ctx.prune_on_equal() && f.rd == md)) continue;
    off[restore_dim] = f.old_off;
    const A best = ctx.max_dist();
    const A rd = f.rd;
    size_t leaf;
    for (;;) {
      if (t.terminal(s.stem_idx, &leaf)) break;
      if (s.level > t.max_stem_level) {
        leaf = t.resolve(s.stem_idx, cursor_leaf(s));
        break;
      }
      if (st) st->stem_visits++;
      const A pivot = s.stem_idx < t.stems.size() ? t.stems[s.stem_idx] : INF;
      if (pivot < INF) {
        const bool is_right = q[dim] >= pivot;
        C far = s.branch_relative(is_right);
        const A new_off = std::fabs(q[dim] - pivot);  // Axis::saturating_dist
        const A rd_far = M::template rect_k<A, K>(rd, off, dim, new_off);
        if (!(rd_far > best)) stack.push_back({far, dim, new_off, rd_far});
      } else {
        s.traverse(false);
      }
      dim = s.dim();
    }
    if (leaf >= t.leaf_count()) continue;  // an unmapped terminal (the reference panics)
    if (st) { st->leaf_visits++; st->points_scanned += t.leaf_len(leaf); }
    process_leaf(leaf);
  }
}

template <typename A, int K, typename M, typename Ctx, typename Leaf>
void scalar_backtracking_query(const Tree<A, K>& t, const A* q, Ctx& ctx, Leaf&& process_leaf,
                               Stats* st) {
  if (t.stem_strategy == 1) {
    DonnellyCursor<K> root;
    root.bh = t.bh;
    scalar_backtracking_query_c<A, K, M>(t, root, q, ctx, process_leaf, st);
  } else {
    scalar_backtracking_query_c<A, K, M>(t, EytzingerCursor<K>(), q, ctx, process_leaf, st);
  }
}

// The traversal the reference runs for this tree (orchestrator/mod.rs:
// 214-255): arithmetic DFS for Eytzinger stems with arithmetic resolution,
// scalar backtracking for Donnelly stems and for Mapped resolution.
template <typename A, int K, typename M, typename Ctx, typename Leaf>
void tree_query(const Tree<A, K>& t, const A* q, Ctx& ctx, Leaf&& process_leaf, Stats* st) {
  if (t.stem_strategy == 1 || t.mapped)
    scalar_backtracking_query<A, K, M>(t, q, ctx, process_leaf, st);
  else
    arithmetic_query<A, K, M>(t, q, ctx, process_leaf, st);
}

// Straight descent (orchestrator/mod.rs:133-178, traits/stem_strategy.rs:182-200);
// Mapped trees stop at a terminal stem (get_leaf_idx_mapped).
template <typename A, int K, typename C>
size_t get_leaf_idx_c(const Tree<A, K>& t, C s, const A* q, Stats* st) {
  size_t leaf;
  while (s.level <= t.max_stem_level) {
    if (t.terminal(s.stem_idx, &leaf)) return leaf;
    if (st) st->stem_visits++;
    const A pivot = s.stem_idx < t.stems.size() ? t.stems[s.stem_idx] : inf_value<A>();
    s.traverse(q[s.dim()] >= pivot);
  }
  return t.resolve(s.stem_idx, cursor_leaf(s));
}
template <typename A, int K>
size_t get_leaf_idx(const Tree<A, K>& t, const A* q, Stats* st) {
  if (t.stem_strategy == 1) {
    DonnellyCursor<K> s;
    s.bh = t.bh;
    return get_leaf_idx_c(t, s, q, st);
  }
  return get_leaf_idx_c(t, EytzingerCursor<K>(), q, st);
}

// ---------------------------------------------------------------------------
// Result collectors (results/result_collection.rs)
// ---------------------------------------------------------------------------
template <typename A>
struct Hit {
  A dist;
  uint32_t item;
  uint64_t seq;  // arrival order
};

// ThresholdVecResultCollection (result_collection.rs:136-215) with a stable
// fill sort: "the k smallest by (distance, arrival)".  Also used for the
// BinaryHeap collector, whose distance multiset (and so threshold) is the same.
template <typename A>
struct TopK {
  size_t k;
  std::vector<Hit<A>> v;   // while filling: arrival order; once full: sorted
  bool sorted = false;
  uint64_t seq = 0;
  explicit TopK(size_t k_) : k(k_) { v.reserve(k_); }
  bool full() const { return v.size() >= k; }
  void add(A d, uint32_t item) {
    Hit<A> h{d, item, seq++};
    if (v.size() < k) {
      v.push_back(h);
      if (v.size() == k) {
        std::stable_sort(v.begin(), v.end(),
                         [](const Hit<A>& a, const Hit<A>& b) { return a.dist < b.dist; });
        sorted = true;
      }
    } else if (d < v[k - 1].dist) {
      size_t i = k - 1;
      while (i > 0 && v[i - 1].dist > d) { v[i] = v[i - 1]; --i; }
      v[i] = h;
    }
  }
  bool threshold(A* out) const {
    if (v.size() == k) { *out = v[k - 1].dist; return true; }
    return false;
  }
  // into_sorted_vec (result_collection.rs:203-214)
  std::vector<Hit<A>> into_sorted() const {
    std::vector<Hit<A>> r = v;
    if (!sorted)
      std::stable_sort(r.begin(), r.end(),
                       [](const Hit<A>& a, const Hit<A>& b) { return a.dist < b.dist; });
    return r;
  }
};

// ---------------------------------------------------------------------------
// Query families
// ---------------------------------------------------------------------------

// nearest_one (kd_tree/query/nearest_one.rs:111-143, ctx :321-352, leaf kernel
// leaf_view_chunked/nearest_one/fallback.rs:69-104)
template <typename A, int K, typename M>
std::pair<A, uint32_t> nearest_one(const Tree<A, K>& t, const A* q, Stats* st) {
  struct Ctx {
    A best;
    A max_dist() const { return best; }
    bool initial_bound_is_unbounded() const { return true; }
    bool prune_on_equal() const { return true; }
  } ctx{inf_value<A>()};
  uint32_t best_item = 0;
  tree_query<A, K, M>(t, q, ctx, [&](size_t leaf) {
    t.for_each_point(leaf, [&](const A* c, uint32_t item) {
      A d = point_dist<M, A, K>(c, q);
      if (d < ctx.best) { ctx.best = d; best_item = item; }
    });
  }, st);
  return {ctx.best, best_item};
}

// approx_nearest_one (kd_tree/query/approx_nearest_one.rs:49-71)
template <typename A, int K, typename M>
std::pair<A, uint32_t> approx_nearest_one(const Tree<A, K>& t, const A* q, Stats* st) {
  A best = inf_value<A>();
  uint32_t best_item = 0;
  if (t.leaf_count() == 0) return {best, best_item};
  size_t leaf = get_leaf_idx(t, q, st);
  if (leaf >= t.leaf_count()) return {best, best_item};
  if (st) { st->leaf_visits++; st->points_scanned += t.leaf_len(leaf); }
  t.for_each_point(leaf, [&](const A* c, uint32_t item) {
    A d = point_dist<M, A, K>(c, q);
    if (d < best) { best = d; best_item = item; }
  });
  return {best, best_item};
}

// nearest_n_within_inner with ThresholdVec/BinaryHeap collectors
// (kd_tree/query/nearest_n_within.rs:127-178, 274-313, ctx :441-479; leaf
// kernel leaf_view_chunked/nearest_n_within/fallback.rs:37-95).
// `unsorted` reproduces into_vec(): arrival order while not full.
template <typename A, int K, typename M>
std::vector<Hit<A>> nearest_n_within(const Tree<A, K>& t, const A* q, A max_dist, size_t k,
                                     bool exclusive, bool sorted, Stats* st) {
  TopK<A> res(k);
  struct Ctx {
    const TopK<A>* res;
    A r;
    bool excl;
    A max_dist() const {
      A cap;
      if (res->threshold(&cap) && cap < r) return cap;
      return r;
    }
    bool initial_bound_is_unbounded() const { return r == inf_value<A>(); }
    bool prune_on_equal() const { return excl; }
  } ctx{&res, max_dist, exclusive};
  tree_query<A, K, M>(t, q, ctx, [&](size_t leaf) {
    const A leaf_max = ctx.max_dist();
    t.for_each_point(leaf, [&](const A* c, uint32_t item) {
      A d = point_dist<M, A, K>(c, q);
      bool ok = exclusive ? (d < leaf_max) : (d <= leaf_max);
      if (ok) res.add(d, item);
    });
  }, st);
  // into_vec() of a ThresholdVec (k <= 24) is arrival order until it fills;
  // every other case is (distance, arrival) order.
  if (sorted || res.sorted || k > 24) return res.into_sorted();
  return res.v;
}

// within / within().unsorted() with the Vec collector
// (kd_tree/query/within.rs:18-41, within_unsorted.rs:133-157;
//  result_collection.rs:1269-1318: sorted = stable sort by distance).
template <typename A, int K, typename M>
std::vector<Hit<A>> within(const Tree<A, K>& t, const A* q, A radius, bool exclusive,
                           bool sorted, Stats* st) {
  std::vector<Hit<A>> out;
  struct Ctx {
    A r;
    bool excl;
    A max_dist() const { return r; }
    bool initial_bound_is_unbounded() const { return r == inf_value<A>(); }
    bool prune_on_equal() const { return excl; }
  } ctx{radius, exclusive};
  uint64_t seq = 0;
  tree_query<A, K, M>(t, q, ctx, [&](size_t leaf) {
    t.for_each_point(leaf, [&](const A* c, uint32_t item) {
      A d = point_dist<M, A, K>(c, q);
      bool ok = exclusive ? (d < radius) : (d <= radius);
      if (ok) out.push_back({d, item, seq++});
    });
  }, st);
  if (sorted)
    std::stable_sort(out.begin(), out.end(),
                     [](const Hit<A>& a, const Hit<A>& b) { return a.dist < b.dist; });
  return out;
}

// best_n_within (kd_tree/query/best_n_within.rs:88-196, ctx :281-306; leaf
// kernel leaf_view_chunked/best_n_within/fallback.rs:40-104; heap
// result_collection.rs:463-560, item order best_query_result_item.rs:27-31).
// Result: the n smallest by (item, arrival), returned in that order.
template <typename A, int K, typename M>
std::vector<Hit<A>> best_n_within(const Tree<A, K>& t, const A* q, A radius, size_t n,
                                  bool exclusive, Stats* st) {
  std::vector<Hit<A>> heap;  // kept sorted by (item, seq)
  struct Ctx {
    A r;
    bool excl;
    A max_dist() const { return r; }
    bool initial_bound_is_unbounded() const { return false; }
    bool prune_on_equal() const { return excl; }
  } ctx{radius, exclusive};
  uint64_t seq = 0;
  auto less = [](const Hit<A>& a, const Hit<A>& b) {
    return a.item < b.item || (a.item == b.item && a.seq < b.seq);
  };
  tree_query<A, K, M>(t, q, ctx, [&](size_t leaf) {
    const bool full_at_entry = heap.size() >= n;
    const uint32_t threshold_item = full_at_entry ? heap.back().item : 0;
    t.for_each_point(leaf, [&](const A* c, uint32_t item) {
      A d = point_dist<M, A, K>(c, q);
      bool ok = exclusive ? (d < radius) : (d <= radius);
      if (!ok) return;
      if (full_at_entry && item >= threshold_item) return;
      Hit<A> h{d, item, seq++};
      if (heap.size() < n) {
        heap.insert(std::upper_bound(heap.begin(), heap.end(), h, less), h);
      } else if (item < heap.back().item) {
        heap.pop_back();
        heap.insert(std::upper_bound(heap.begin(), heap.end(), h, less), h);
      }
    });
  }, st);
  return heap;
}

// ---------------------------------------------------------------------------
// Periodic boundary conditions (kd_tree/query/periodic.rs)
// ---------------------------------------------------------------------------

// periodic_image_axis_offset (periodic.rs:29-37)
template <typename A>
inline A image_axis_offset(A wrapped, A axis_len) {
  if (wrapped < A(0)) return std::fabs(wrapped - A(0));
  if (wrapped > axis_len) return std::fabs(wrapped - axis_len);
  return A(0);
}

template <typename A, int K>
struct ImageCandidate {
  A wrapped[K];
  A lower_bound;
};

// periodic_image_candidates (periodic.rs:45-142), threshold Exclusive.
template <typename A, int K, typename M>
void image_candidates_rec(const A* q, const A* box, int axis, A* wrapped, bool nonzero, A lb,
                          A limit, std::vector<ImageCandidate<A, K>>& out) {
  if (axis == K) {
    if (nonzero) {
      ImageCandidate<A, K> c;
      for (int d = 0; d < K; ++d) c.wrapped[d] = wrapped[d];
      c.lower_bound = lb;
      out.push_back(c);
    }
    return;
  }
  const A original = q[axis];
  const A L = box[axis];
  for (int shift = -1; shift <= 1; ++shift) {
    A w = shift == -1 ? original - L : (shift == 0 ? original : original + L);
    wrapped[axis] = w;
    A offset = image_axis_offset(w, L);
    A next = M::combine(lb, M::template dist1<A>(offset, A(0)));
    if (!(next < limit)) continue;  // boundary_accepts(Exclusive, next, limit)
    image_candidates_rec<A, K, M>(q, box, axis + 1, wrapped, nonzero || shift != 0, next, limit,
                                  out);
  }
  wrapped[axis] = original;
}

// periodic_nearest_one_result (periodic.rs:156-214)
template <typename A, int K, typename M>
std::pair<A, uint32_t> periodic_nearest_one(const Tree<A, K>& t, const A* q, const A* box,
                                            Stats* st) {
  auto home = nearest_one<A, K, M>(t, q, st);
  A best = home.first;
  uint32_t best_item = home.second;
  std::vector<ImageCandidate<A, K>> cands;
  A wrapped[K];
  for (int d = 0; d < K; ++d) wrapped[d] = q[d];
  image_candidates_rec<A, K, M>(q, box, 0, wrapped, false, A(0), best, cands);
  std::stable_sort(cands.begin(), cands.end(),
                   [](const ImageCandidate<A, K>& a, const ImageCandidate<A, K>& b) {
                     return a.lower_bound < b.lower_bound;
                   });
  for (const auto& c : cands) {
    if (!(c.lower_bound < best)) continue;
    auto r = nearest_one<A, K, M>(t, c.wrapped, st);
    if (r.first < best) { best = r.first; best_item = r.second; }
  }
  return {best, best_item};
}

// interval_distance_1d (stem_strategy/donnelly/simd_full/mod.rs:209-216)
template <typename A>
inline A interval_distance_1d(A q, A lo, A hi) {
  A below = std::max(A(0), lo - q);
  A above = std::max(A(0), q - hi);
  return below + above;
}

// periodic_interval_distance_1d (periodic.rs:286-308)
template <typename A>
inline A periodic_interval_distance_1d(A q, A lo, A hi, A L) {
  A best = interval_distance_1d(q, lo, hi);
  A minus = interval_distance_1d(q, lo - L, hi - L);
  if (minus < best) best = minus;
  A lp = lo; lp += L;
  A hp = hi; hp += L;
  A plus = interval_distance_1d(q, lp, hp);
  if (plus < best) best = plus;
  return best;
}

// periodic_min_image_axis_delta (periodic.rs:272-284)
template <typename A>
inline A min_image_delta(A q, A c, A L) {
  A delta = std::fabs(q - c);
  A wrapped = L - delta;
  return wrapped < delta ? wrapped : delta;
}

// periodic_backtracking_query (periodic.rs:455-619) driving a collector
// through `max_dist()`, `prune_on_equal()` and `leaf(leaf_idx)`, over the
// stem order of cursor C (EytzingerCursor or DonnellyCursor: periodic.rs
// drives both through the StemStrategy trait).  A far child is pushed unless pruned when it is
// generated; popped frames are not tested again.
template <typename A, int K, typename M, typename C, typename Ctx, typename Leaf>
void periodic_query_c(const Tree<A, K>& t, C root, const A* q, const A* box, Ctx& ctx,
                      Leaf&& leaf_fn, Stats* st) {
  if (t.size == 0) return;
  struct Frame { C s; A lower[K]; A upper[K]; A off[K]; A rd; };
  std::vector<Frame> stack;
  C s = root;
  A lower[K], upper[K], off[K];
  for (int d = 0; d < K; ++d) { lower[d] = A(0); upper[d] = box[d]; off[d] = A(0); }
  A rd = A(0);
  const A INF = inf_value<A>();
  auto pop = [&]() -> bool {
    if (stack.empty()) return false;
    Frame f = stack.back();
    stack.pop_back();
    s = f.s; rd = f.rd;
    for (int d = 0; d < K; ++d) { lower[d] = f.lower[d]; upper[d] = f.upper[d]; off[d] = f.off[d]; }
    return true;
  };
  for (;;) {
    bool finished = false;
    for (;;) {
      // resolve_terminal_stem, then the walk past max_stem_level (periodic.rs:496-510)
      size_t leaf;
      bool at_leaf = t.terminal(s.stem_idx, &leaf);
      if (!at_leaf && s.level > t.max_stem_level) {
        leaf = t.resolve(s.stem_idx, cursor_leaf(s));
        at_leaf = true;
      }
      if (at_leaf) {
        if (leaf < t.leaf_count()) {
          if (st) { st->leaf_visits++; st->points_scanned += t.leaf_len(leaf); }
          leaf_fn(leaf);
        }
        break;
      }
      if (st) st->stem_visits++;
      const int dim = s.dim();
      const A pivot = s.stem_idx < t.stems.size() ? t.stems[s.stem_idx] : INF;
      if (pivot >= INF) { s.traverse(false); continue; }
      const A old_lower = lower[dim], old_upper = upper[dim];
      const bool is_right = q[dim] >= pivot;
      C far = s.branch_relative(is_right);
      const A minup = old_upper < pivot ? old_upper : pivot;
      const A maxlo = std::max(old_lower, pivot);
      A near_lo, near_hi, far_lo, far_hi;
      if (is_right) { near_lo = maxlo; near_hi = old_upper; far_lo = old_lower; far_hi = minup; }
      else { near_lo = old_lower; near_hi = minup; far_lo = maxlo; far_hi = old_upper; }
      const A near_off = periodic_interval_distance_1d(q[dim], near_lo, near_hi, box[dim]);
      const A far_off = periodic_interval_distance_1d(q[dim], far_lo, far_hi, box[dim]);
      const A near_rd = M::template rect_k<A, K>(rd, off, dim, near_off);
      const A far_rd = M::template rect_k<A, K>(rd, off, dim, far_off);
      const A thr = ctx.max_dist();
      const bool poe = ctx.prune_on_equal();
      const bool near_pruned = near_rd > thr || (poe && near_rd == thr);
      const bool far_pruned = far_rd > thr || (poe && far_rd == thr);
      if (!far_pruned) {
        Frame f;
        f.s = far; f.rd = far_rd;
        for (int d = 0; d < K; ++d) { f.lower[d] = lower[d]; f.upper[d] = upper[d]; f.off[d] = off[d]; }
        f.lower[dim] = far_lo; f.upper[dim] = far_hi; f.off[dim] = far_off;
        stack.push_back(f);
      }
      if (near_pruned) {
        if (pop()) continue;
        finished = true;
        break;
      }
      lower[dim] = near_lo; upper[dim] = near_hi; off[dim] = near_off; rd = near_rd;
    }
    if (finished) return;
    if (!pop()) return;
  }
}

// periodic_query over the tree's own stem order.
template <typename A, int K, typename M, typename Ctx, typename Leaf>
void periodic_query(const Tree<A, K>& t, const A* q, const A* box, Ctx& ctx, Leaf&& leaf_fn,
                    Stats* st) {
  if (t.stem_strategy == 1) {
    DonnellyCursor<K> root;
    root.bh = t.bh;
    periodic_query_c<A, K, M>(t, root, q, box, ctx, leaf_fn, st);
  } else {
    periodic_query_c<A, K, M>(t, EytzingerCursor<K>(), q, box, ctx, leaf_fn, st);
  }
}

// periodic leaf distance (process_periodic_leaf_arena, periodic.rs:357-400):
// combine_component over the min-image components, from zero
template <typename A, int K, typename M>
inline A periodic_point_dist(const A* c, const A* q, const A* box) {
  A acc = A(0);
  for (int d = 0; d < K; ++d) {
    A delta = min_image_delta(q[d], c[d], box[d]);
    acc = M::combine(acc, M::template dist1<A>(delta, A(0)));
  }
  return acc;
}

// periodic_nearest_results (periodic.rs:682-791): radius and/or max_qty.
// k == 0 means "no max_qty" (Vec collector).
template <typename A, int K, typename M>
std::vector<Hit<A>> periodic_nearest(const Tree<A, K>& t, const A* q, const A* box, A radius,
                                     size_t k, bool exclusive, bool sorted, Stats* st) {
  if (k == 0) {
    std::vector<Hit<A>> out;
    struct Ctx {
      A r; bool excl;
      A max_dist() const { return r; }
      bool prune_on_equal() const { return excl; }
    } ctx{radius, exclusive};
    uint64_t seq = 0;
    periodic_query<A, K, M>(t, q, box, ctx, [&](size_t leaf) {
      t.for_each_point(leaf, [&](const A* c, uint32_t item) {
        A d = periodic_point_dist<A, K, M>(c, q, box);
        bool ok = exclusive ? (d < radius) : (d <= radius);
        if (ok) out.push_back({d, item, seq++});
      });
    }, st);
    if (sorted)
      std::stable_sort(out.begin(), out.end(),
                       [](const Hit<A>& a, const Hit<A>& b) { return a.dist < b.dist; });
    return out;
  }
  TopK<A> res(k);
  struct Ctx {
    const TopK<A>* res; A r; bool excl;
    A max_dist() const {
      A cap;
      if (res->threshold(&cap) && cap < r) return cap;
      return r;
    }
    bool prune_on_equal() const { return excl; }
  } ctx{&res, radius, exclusive};
  periodic_query<A, K, M>(t, q, box, ctx, [&](size_t leaf) {
    const A leaf_max = ctx.max_dist();
    t.for_each_point(leaf, [&](const A* c, uint32_t item) {
      A d = periodic_point_dist<A, K, M>(c, q, box);
      bool ok = exclusive ? (d < leaf_max) : (d <= leaf_max);
      if (ok) res.add(d, item);
    });
  }, st);
  // ThresholdVec (sorted, k <= 20) and BinaryHeap (every other case) both
  // hold the k smallest; output is (distance, arrival) order.
  (void)sorted;
  return res.into_sorted();
}

}  // namespace kiddo_oracle
