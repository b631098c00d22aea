// layout_build.cpp — host construction of the ImmutableKdTree layout.
//
// Produces the exact bytes kiddo's soft-bucket bulk construction writes for
// KdTree<A, u32, Eytzinger, VecOfArenas<A, u32, K, 32>, K, 32>:
//   new_from_source_with        src/kd_tree/construction.rs:413-539
//   populate_recursive_soft     src/kd_tree/construction.rs:868-968
//   soft_left_leaf_budget/ideal src/kd_tree/construction.rs:673-691
//   update_pivot                src/kd_tree/construction.rs:1089-1175
//   VecOfArenas::append_leaf    src/leaf_strategy/vec_of_arenas.rs:292-323
//
// Design: the partition works on a u32 index permutation over per-axis
// coordinate columns; subtrees below the top levels are built concurrently;
// each leaf only records its index range during the recursion, and the arena
// is written afterwards in one parallel pass once leaf offsets are known.  The
// pivot rule is the reference's (the nudge-left / nudge-right of
// update_pivot expressed as counts around the k-th order statistic), so stem
// values and leaf membership match the reference exactly; points inside a
// leaf are stored in ascending source index.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <new>
#include <stdexcept>
#include <thread>
#include <vector>

#include "kgpu_internal.h"

namespace kgpu {

namespace {

constexpr size_t kB = 32;

inline size_t tile_width(size_t remaining) {
  if (remaining >= 32) return 32;
  if (remaining >= 8) return 8;
  if (remaining >= 4) return 4;
  if (remaining >= 2) return 2;
  return 1;
}

template <typename A>
size_t leaf_encoded_bytes(size_t len, int K) {
  size_t total = 0;
  while (len) {
    size_t w = tile_width(len);
    total += w * (K * sizeof(A) + sizeof(uint32_t));
    len -= w;
  }
  return total;
}

// Position of a node in the stem tree: its stem index, level, split
// dimension, arithmetic leaf prefix (the path bits), and for Donnelly stems its
// level inside the current minor triangle.
struct NodePos {
  uint32_t stem = 1;
  int level = 0;
  uint32_t minor = 0;
  uint64_t leaf = 0;
  int dim = 0;
};

// Children of a node.  bh == 0: Eytzinger (children 2i and 2i + 1,
// stem_strategy/eytzinger/mod.rs:131-168).  bh > 0: Donnelly<bh>
// (stem_strategy/donnelly/core.rs:400-428): inside a minor triangle the
// children are 2m + 1 and 2m + 2 of the line's heap; from the triangle's
// bottom row they are the roots of lines (base + 1 + 2(m - minor - 1) + side)
// << bh.  The dimension advances once per level in both.
inline void node_children(const NodePos& n, int K, uint32_t bh, NodePos& l, NodePos& r) {
  l = n;
  l.level = n.level + 1;
  l.leaf = n.leaf << 1;
  l.dim = n.dim + 1 == K ? 0 : n.dim + 1;
  r = l;
  r.leaf = l.leaf | 1u;
  if (!bh) {
    l.stem = n.stem * 2u;
    r.stem = l.stem + 1u;
    return;
  }
  const uint32_t mask = (1u << bh) - 1u;
  const uint32_t min_idx = n.stem & mask;
  const uint32_t base = (n.stem & ~mask) + 1u;
  if (n.minor + 1u == bh) {
    l.stem = (base + ((min_idx - n.minor - 1u) << 1)) << bh;
    r.stem = l.stem + (1u << bh);
    l.minor = r.minor = 0;
  } else {
    l.stem = base + (min_idx << 1);
    r.stem = l.stem + 1u;
    l.minor = r.minor = n.minor + 1u;
  }
}

template <typename A>
struct SoftBuilder {
  int K;
  uint32_t bh = 0;  // 0: Eytzinger stems; 3 or 4: Donnelly<bh>
  std::vector<std::vector<A>> cols;   // cols[d][i]
  uint32_t* idx;
  A* stems;
  int max_stem_level;
  uint32_t depth;
  std::vector<uint64_t>* leaf_begin;  // per leaf: begin offset into idx
  std::vector<uint32_t>* leaf_len;
  int spawn_levels;
  int root_level = 0;

  // Reference pivot rule (update_pivot) for chunk idx[b, e) on `dim`.
  // Returns the pivot and the split value t (left = x < t) and the stem value.
  size_t choose_pivot(uint32_t* b, size_t len, int dim, size_t ideal, std::vector<A>& buf,
                      A* split_value) {
    const A* col = cols[dim].data();
    buf.resize(len);
    for (size_t i = 0; i < len; ++i) buf[i] = col[b[i]];
    std::nth_element(buf.begin(), buf.begin() + ideal, buf.end());
    const A v = buf[ideal];
    size_t lt = 0, le = 0;
    A above = std::numeric_limits<A>::infinity();
    for (size_t i = 0; i < len; ++i) {
      const A x = buf[i];
      lt += x < v;
      le += x <= v;
      if (x > v && x < above) above = x;
    }
    if (lt > 0) { *split_value = v; return lt; }
    if (le >= len) { *split_value = v; return len; }
    *split_value = above;  // left = {x <= v} = {x < above}
    return le;
  }

  void build(uint32_t* b, size_t len, NodePos root, uint64_t budget, uint64_t base) {
    std::vector<A> buf;
    build_rec(b, len, root, budget, base, buf);
  }

  void build_rec(uint32_t* b, size_t len, NodePos node, uint64_t budget, uint64_t base,
                 std::vector<A>& buf) {
    if (budget == 0) return;
    const int level = node.level;
    const uint32_t stem_idx = node.stem;
    if (level > max_stem_level) {
      const uint64_t leaf = node.leaf;
      (*leaf_begin)[leaf] = base;
      (*leaf_len)[leaf] = uint32_t(len);
      std::sort(b, b + len);
      return;
    }
    const int dim = node.dim;
    uint64_t left_budget, right_budget;
    size_t pivot;
    A split = A(0);
    if (budget == 1) {
      left_budget = 1;
      right_budget = 0;
      pivot = len;
    } else {
      left_budget = uint64_t(1) << (63 - __builtin_clzll(budget - 1));
      right_budget = budget - left_budget;
      if (len == 0) {
        pivot = 0;
      } else {
        unsigned __int128 num = (unsigned __int128)len * left_budget;
        size_t p = size_t((num + budget - 1) / budget);
        pivot = std::min(std::max<size_t>(p, 1), len);
      }
      if (pivot < len) pivot = choose_pivot(b, len, dim, pivot, buf, &split);
    }
    if (pivot < len) {
      const A* col = cols[dim].data();
      std::partition(b, b + len, [&](uint32_t i) { return col[i] < split; });
      stems[stem_idx] = split;  // smallest coordinate of the right part
    }
    const size_t cut = std::min(pivot, len);
    NodePos left, right;
    node_children(node, K, bh, left, right);
    if (level - root_level < spawn_levels && len > 65536) {
      std::thread th([&, b, cut, left, left_budget, base]() {
        std::vector<A> buf2;
        build_rec(b, cut, left, left_budget, base, buf2);
      });
      build_rec(b + cut, len - cut, right, right_budget, base + cut, buf);
      th.join();
    } else {
      build_rec(b, cut, left, left_budget, base, buf);
      build_rec(b + cut, len - cut, right, right_budget, base + cut, buf);
    }
  }
};

template <typename F>
void parallel_range(size_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 4096) {
    f(size_t(0), n);
    return;
  }
  std::vector<std::thread> th;
  const size_t per = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; ++t) {
    size_t b = t * per, e = std::min(n, b + per);
    if (b >= e) break;
    th.emplace_back([&, b, e]() { f(b, e); });
  }
  for (auto& x : th) x.join();
}

template <typename A>
void write_leaf(uint8_t* dst, const A* pts, const uint32_t* items, const uint32_t* idx,
                size_t len, int K) {
  size_t off = 0, base = 0;
  while (len) {
    const size_t w = tile_width(len);
    for (int d = 0; d < K; ++d) {
      A* col = reinterpret_cast<A*>(dst + off + d * w * sizeof(A));
      for (size_t i = 0; i < w; ++i) col[i] = pts[size_t(idx[base + i]) * K + d];
    }
    uint32_t* it = reinterpret_cast<uint32_t*>(dst + off + K * w * sizeof(A));
    for (size_t i = 0; i < w; ++i) it[i] = items ? items[idx[base + i]] : idx[base + i];
    off += w * (K * sizeof(A) + sizeof(uint32_t));
    base += w;
    len -= w;
  }
}

template <typename A>
void build_layout(Layout& L, const A* pts, const uint32_t* items, uint64_t n, int K,
                  uint32_t bh, int nthreads) {
  L.block_height = bh;
  L.dtype = sizeof(A) == 8 ? 1 : 0;
  L.dims = K;
  L.size = n;
  L.max_stem_level = -1;
  L.max_leaf_len = 0;
  L.stems_bytes.clear();
  L.leaf_bytes.clear();
  L.extents.clear();
  if (n == 0) return;
  const uint64_t leaf_node_count = (n + kB - 1) / kB;
  std::vector<uint32_t> idx(n);
  for (uint64_t i = 0; i < n; ++i) idx[i] = uint32_t(i);

  std::vector<uint64_t> leaf_begin;
  std::vector<uint32_t> leaf_len;
  if (leaf_node_count < 2) {
    leaf_begin.assign(1, 0);
    leaf_len.assign(1, uint32_t(n));
  } else {
    uint32_t depth = 0;
    while ((uint64_t(1) << depth) < leaf_node_count) ++depth;
    const uint32_t leaf_bits = depth;
    // Block strategies pad the stem tree at the root to a multiple of bh
    // levels; the padding levels are walked to the left (construction.rs:
    // 431-446) and carry no stems.
    const uint32_t pad = bh && depth % bh ? bh - depth % bh : 0;
    depth += pad;
    NodePos root;
    root.stem = bh ? 0u : 1u;  // Eytzinger root 1, Donnelly root 0
    for (uint32_t i = 0; i < pad; ++i) {
      NodePos l, r;
      node_children(root, K, bh, l, r);
      root = l;
    }
    const uint64_t budget = uint64_t(1) << depth;
    // stem count: the index of the node reached by walking `depth` levels to
    // the right from the root, plus one, padded to 8 (construction.rs:448-469)
    NodePos far_right = root;
    for (uint32_t i = 0; i < depth; ++i) {
      NodePos l, r;
      node_children(far_right, K, bh, l, r);
      far_right = r;
    }
    const size_t stem_count = size_t(far_right.stem) + 1;
    const size_t padded = (stem_count + 7) / 8 * 8;
    L.stems_bytes.resize(padded * sizeof(A));
    A* stems = reinterpret_cast<A*>(L.stems_bytes.data());
    for (size_t i = 0; i < padded; ++i) stems[i] = std::numeric_limits<A>::infinity();
    leaf_begin.assign(uint64_t(1) << leaf_bits, 0);
    leaf_len.assign(uint64_t(1) << leaf_bits, 0);

    SoftBuilder<A> sb;
    sb.K = K;
    sb.cols.resize(K);
    for (int d = 0; d < K; ++d) sb.cols[d].resize(n);
    parallel_range(n, nthreads, [&](size_t b, size_t e) {
      for (size_t i = b; i < e; ++i)
        for (int d = 0; d < K; ++d) sb.cols[d][i] = pts[i * K + d];
    });
    sb.idx = idx.data();
    sb.stems = stems;
    sb.max_stem_level = int(depth) - 1;
    sb.depth = depth;
    sb.leaf_begin = &leaf_begin;
    sb.leaf_len = &leaf_len;
    int spawn = 0;
    while ((1 << spawn) < std::max(1, nthreads)) ++spawn;
    sb.spawn_levels = spawn + 1;
    sb.bh = bh;
    sb.root_level = root.level;
    sb.build(idx.data(), n, root, budget, 0);
    L.max_stem_level = int(depth) - 1;
  }
  if (leaf_node_count < 2) std::sort(idx.begin(), idx.end());

  // Arena offsets: each leaf starts on max(align A, align u32, 8) bytes.
  const size_t nleaves = leaf_len.size();
  L.extents.resize(2 * nleaves);
  uint64_t cursor = 0;
  for (size_t l = 0; l < nleaves; ++l) {
    cursor = (cursor + 7) & ~uint64_t(7);
    L.extents[2 * l] = cursor;
    L.extents[2 * l + 1] = leaf_len[l];
    cursor += leaf_encoded_bytes<A>(leaf_len[l], K);
    L.max_leaf_len = std::max<uint64_t>(L.max_leaf_len, leaf_len[l]);
  }
  L.leaf_bytes.assign(cursor, 0);
  parallel_range(nleaves, nthreads, [&](size_t b, size_t e) {
    for (size_t l = b; l < e; ++l)
      write_leaf<A>(L.leaf_bytes.data() + L.extents[2 * l], pts, items, idx.data() + leaf_begin[l],
                    leaf_len[l], K);
  });
}

}  // namespace

namespace {

// FlatVec leaves (leaf_strategy/flat_vec.rs:20-26, 189-210) re-encoded in the
// VecOfArenas tiles: leaf l holds points start..end of the K columns, in that
// order, the same chunk VecOfArenas::append_leaf would have been given.
template <typename A>
void flatvec_arena(Layout& L, const void* const* columns, const uint32_t* items,
                   const uint32_t* ext, uint64_t leaf_count, int K) {
  L.extents.resize(2 * leaf_count);
  uint64_t cursor = 0;
  for (uint64_t l = 0; l < leaf_count; ++l) {
    const uint64_t len = ext[2 * l + 1] - ext[2 * l];
    cursor = (cursor + 7) & ~uint64_t(7);
    L.extents[2 * l] = cursor;
    L.extents[2 * l + 1] = len;
    cursor += leaf_encoded_bytes<A>(len, K);
    L.max_leaf_len = std::max<uint64_t>(L.max_leaf_len, len);
  }
  L.leaf_bytes.assign(cursor, 0);
  for (uint64_t l = 0; l < leaf_count; ++l) {
    uint8_t* dst = L.leaf_bytes.data() + L.extents[2 * l];
    size_t len = L.extents[2 * l + 1], base = ext[2 * l], off = 0;
    while (len) {
      const size_t w = tile_width(len);
      for (int d = 0; d < K; ++d) {
        const A* src = static_cast<const A*>(columns[d]) + base;
        std::memcpy(dst + off + d * w * sizeof(A), src, w * sizeof(A));
      }
      std::memcpy(dst + off + K * w * sizeof(A), items + base, w * sizeof(uint32_t));
      off += w * (K * sizeof(A) + sizeof(uint32_t));
      base += w;
      len -= w;
    }
  }
}

}  // namespace

int flatvec_to_layout(Layout& L, int dtype, int K, const void* const* columns,
                      const uint32_t* items, const uint32_t* extents, uint64_t leaf_count,
                      uint64_t size) {
  if (K < 1 || K > kMaxDims) return set_error(KGPU_EUNSUPPORTED, "dims must be 1..4");
  if (dtype != KGPU_F32 && dtype != KGPU_F64)
    return set_error(KGPU_EINVAL, "dtype must be KGPU_F32 or KGPU_F64");
  if (size > 0xFFFFFFFFull) return set_error(KGPU_EOVERFLOW, "more than 2^32 points");
  if (size > 0) {
    if (!items) return set_error(KGPU_EINVAL, "leaf_items is NULL");
    for (int d = 0; d < K; ++d)
      if (!columns[d]) return set_error(KGPU_EINVAL, "a leaf_points column is NULL");
  }
  if (leaf_count > 0 && !extents) return set_error(KGPU_EINVAL, "leaf_extents is NULL");
  uint64_t total = 0;
  for (uint64_t l = 0; l < leaf_count; ++l) {
    const uint32_t a = extents[2 * l], b = extents[2 * l + 1];
    if (a > b || b > size) return set_error(KGPU_EINVAL, "leaf extent outside the points");
    if (b - a > 1024) return set_error(KGPU_EINVAL, "leaf longer than 1024 points");
    total += b - a;
  }
  if (total != size) return set_error(KGPU_EINVAL, "sum of leaf lengths != size");
  L.dtype = dtype == KGPU_F64 ? 1 : 0;
  L.dims = K;
  L.size = size;
  L.max_leaf_len = 0;
  try {
    if (dtype == KGPU_F32)
      flatvec_arena<float>(L, columns, items, extents, leaf_count, K);
    else
      flatvec_arena<double>(L, columns, items, extents, leaf_count, K);
  } catch (const std::bad_alloc&) {
    return set_error(KGPU_ENOMEM, "host allocation failed");
  }
  return KGPU_OK;
}

int build_layout_any(Layout& L, int dtype, int K, const void* pts, const uint32_t* items,
                     uint64_t n, int nthreads, uint32_t block_height) {
  if (K < 1 || K > kMaxDims) return set_error(KGPU_EUNSUPPORTED, "dims must be 1..4");
  if (block_height != 0 && block_height != 3 && block_height != 4)
    return set_error(KGPU_EUNSUPPORTED, "Donnelly block height must be 3 or 4");
  if (n > 0 && !pts) return set_error(KGPU_EINVAL, "points is NULL");
  if (n > 0xFFFFFFFFull) return set_error(KGPU_EOVERFLOW, "more than 2^32 points");
  if (nthreads <= 0) nthreads = int(std::max(1u, std::thread::hardware_concurrency()));
  try {
    if (dtype == KGPU_F32)
      build_layout<float>(L, static_cast<const float*>(pts), items, n, K, block_height, nthreads);
    else if (dtype == KGPU_F64)
      build_layout<double>(L, static_cast<const double*>(pts), items, n, K, block_height,
                           nthreads);
    else
      return set_error(KGPU_EINVAL, "dtype must be KGPU_F32 or KGPU_F64");
  } catch (const std::bad_alloc&) {
    return set_error(KGPU_ENOMEM, "host allocation failed while building the layout");
  }
  if (L.max_leaf_len > 1024)
    return set_error(KGPU_EOVERFLOW,
                     "a leaf holds more than 1024 points (leaf scratch capacity, "
                     "leaf_view/mod.rs:18,58-65)");
  return KGPU_OK;
}

}  // namespace kgpu
