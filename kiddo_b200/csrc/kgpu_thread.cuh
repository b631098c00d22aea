// kgpu_thread.cuh — per-thread traversal of the thread-per-query engine.
//
// The warp-per-query kernels spend most issue slots on 32 lanes running the
// same scalar traversal.  Here every thread walks one query's tree, exactly
// in the reference's order (kd_tree/orchestrator/mod.rs:388-603), so a warp
// advances 32 walks per instruction; the leaves they reach are scanned by the
// whole warp (kgpu_coop.cuh).
//
// Continuation state per level L, in shared memory column `slot[L * stride]`:
//  * while the far child of level L is pending: its rd_far;
//  * once the far child has been entered: the off[dim] value to restore on the
//    way back up (the reference's restore frame);
// two bitmasks say which.  A level that never branched needs neither: along a
// near path `off` does not change, so restoring it is a no-op.  far_off is
// recomputed from the stem when the far child is entered (|q - pivot|, the
// same operation the descent did).  Same visit order, same rd arithmetic, same
// results as the per-level restore/far stacks of the reference.
#pragma once

#include <type_traits>

#include "kgpu_device.cuh"

namespace kgpu {

// Sequential tile walk of one leaf (LeafArena::for_each_tiled_chunk,
// leaf_view/mod.rs:431-446) calling f(distance, item) in tile order, with
// distance = dist(coords); pairs where pass() rejects both points skip f.
// Tiles of width >= 2 are read two points per step (8-byte aligned pairs for
// f32: leaves start on 8 bytes and every column of an even-width tile spans
// an even number of floats).  Items are read only for points that reach f, and
// both points of a pair go through one call site of f, so the policy's
// insertion code is emitted once.
template <typename A, int K, typename D, typename P, typename F>
__device__ __forceinline__ uint32_t thread_for_each_point(const TreeView<A>& tv, uint2 ex,
                                                          const D& dist, P&& pass, F&& f) {
  constexpr uint32_t per = K * sizeof(A) + sizeof(uint32_t);
  const uint8_t* base = tv.arena + size_t(ex.x) * 8;
  if constexpr (RowLeaves<A, K>::value) {
    // rows: one row per step, the leaf's lines requested up front
    for (uint32_t b = 0; b < ex.y * row_bytes<A>(); b += 128u)
      asm volatile("prefetch.global.L1 [%0];" ::"l"(base + b));
    for (uint32_t p = 0; p < ex.y; ++p) {
      A c[K];
      uint32_t it;
      load_row<A, K>(base, p, c, it);
      const A d0 = dist(c);
      if (pass(d0)) f(d0, it);
    }
    return ex.y;
  }
  uint32_t rem = ex.y;
  uint32_t boff = 0, i = 0;
  uint32_t w = rem >= 32 ? 32 : rem >= 8 ? 8 : rem >= 4 ? 4 : rem >= 2 ? 2 : 1;
  // one flat loop step per pair; the next tile is taken in a short tail
  while (rem) {
    const A* col = reinterpret_cast<const A*>(base + boff);
    A d0, d1;
    if (w == 1) {
      A c0[K];
#pragma unroll
      for (int d = 0; d < K; ++d) c0[d] = __ldg(col + d);
      d0 = d1 = dist(c0);
    } else if constexpr (sizeof(A) == 4) {
      float2 v[K];
#pragma unroll
      for (int d = 0; d < K; ++d) v[d] = __ldg(reinterpret_cast<const float2*>(col + d * w + i));
      dist.pair(v, d0, d1);
    } else {
      A c0[K], c1[K];
#pragma unroll
      for (int d = 0; d < K; ++d) {
        c0[d] = __ldg(col + d * w + i);
        c1[d] = __ldg(col + d * w + i + 1);
      }
      d0 = dist(c0);
      d1 = dist(c1);
    }
    // `pass` is a cheap necessary condition for f to act: most points fail
    // it once a list has filled, and then f is not entered at all.
    if (pass(d0) || (w > 1 && pass(d1))) {
      const uint32_t* its = reinterpret_cast<const uint32_t*>(base + boff + K * w * sizeof(A));
      const int nu = w == 1 ? 1 : 2;
#pragma unroll 1
      for (int u = 0; u < nu; ++u) f(u ? d1 : d0, __ldg(its + i + u));
    }
    i += 2;
    if (i >= w) {
      boff += w * per;
      rem -= w;
      w = rem >= 32 ? 32 : rem >= 8 ? 8 : rem >= 4 ? 4 : rem >= 2 ? 2 : 1;
      i = 0;
    }
  }
  return ex.y;
}

// Bit j of the result: point c0 + j of the leaf passes pass(distance).  A
// chunk is one 32-point tile (c0 below len & ~31) or the leaf's remainder
// tiles (widths 8, 4, 2, 1).  One flat loop step per pair of points (tiles of
// width >= 2 are read in 8-byte aligned pairs, as in thread_for_each_point),
// moving to the next tile in a short tail, so lanes whose leaves have
// different tile shapes still run the same loop body; nothing but the mask
// depends on the distances.
template <typename A, int K, typename D, typename P>
__device__ __forceinline__ uint32_t leaf_chunk_mask(const uint8_t* __restrict__ base, uint32_t len,
                                                    uint32_t c0, const D& dist, P&& pass) {
  constexpr uint32_t per = K * sizeof(A) + sizeof(uint32_t);
  if constexpr (RowLeaves<A, K>::value) {
    const uint32_t end = len < c0 + 32 ? len : c0 + 32;
    uint32_t mask = 0;
    for (uint32_t p = c0; p < end; ++p) {
      A c[K];
      uint32_t it;
      load_row<A, K>(base, p, c, it);
      if (pass(dist(c))) mask |= 1u << (p - c0);
    }
    return mask;
  }
  const uint32_t full = len & ~31u;
  uint32_t boff, rem;
  if (c0 < full) {
    boff = (c0 >> 5) * (32 * per);
    rem = 32;
  } else {
    boff = full * per;
    rem = len - full;
  }
  uint32_t mask = 0, bit = 0, i = 0;
  uint32_t w = rem >= 32 ? 32 : rem >= 8 ? 8 : rem >= 4 ? 4 : rem >= 2 ? 2 : 1;
  while (rem) {
    const A* col = reinterpret_cast<const A*>(base + boff);
    A d0, d1;
    if (w == 1) {
      A c[K];
#pragma unroll
      for (int d = 0; d < K; ++d) c[d] = __ldg(col + d);
      d0 = d1 = dist(c);
    } else if constexpr (sizeof(A) == 4) {
      float2 v[K];
#pragma unroll
      for (int d = 0; d < K; ++d) v[d] = __ldg(reinterpret_cast<const float2*>(col + d * w + i));
      dist.pair(v, d0, d1);
    } else {
      A c0v[K], c1v[K];
#pragma unroll
      for (int d = 0; d < K; ++d) {
        c0v[d] = __ldg(col + d * w + i);
        c1v[d] = __ldg(col + d * w + i + 1);
      }
      d0 = dist(c0v);
      d1 = dist(c1v);
    }
    mask |= ((pass(d0) ? 1u : 0u) | ((w > 1 && pass(d1)) ? 2u : 0u)) << (bit + i);
    i += 2;
    if (i >= w) {
      boff += w * per;
      bit += w;
      rem -= w;
      w = rem >= 32 ? 32 : rem >= 8 ? 8 : rem >= 4 ? 4 : rem >= 2 ? 2 : 1;
      i = 0;
    }
  }
  return mask;
}

// Resumable traversal state of one query: the reference's DFS
// (kd_tree/orchestrator/mod.rs:388-603) cut at its leaves, so a thread can
// stop after any leaf and carry on later.  descend() runs from the current
// position to the next leaf; backtrack() climbs until a pending far child
// survives the prune test (and enters it) or the root is passed.
template <typename A, int K, typename M>
struct ThreadWalk {
  A off[K];
  A rd;
  uint32_t stem_idx, pending, taken;
  int level, dim, cur;

  __device__ __forceinline__ void init() {
#pragma unroll
    for (int d = 0; d < K; ++d) off[d] = A(0);
    rd = A(0);
    stem_idx = 1;
    pending = taken = 0;
    level = dim = cur = 0;
  }

  template <typename P>
  __device__ __forceinline__ uint32_t descend(const TreeView<A>& tv, const A (&q)[K], const P& pol,
                                              bool check_bound, A* __restrict__ slot, int stride,
                                              TravStats& st) {
    const A INF = inf_of<A>();
    const int msl = tv.max_stem_level;
    while (level <= msl) {
      ++st.stems;
      const A pivot = __ldg(tv.stems + stem_idx);
      if (pivot < INF) {
        const A qd = sel(q, dim);
        const bool is_right = qd >= pivot;
        const A new_off = abs_val(sub_rn(qd, pivot));
        const A rd_far = M::template rect_k<A, K>(rd, off, dim, new_off);
        if (!check_bound || !(rd_far > pol.max_dist())) {
          slot[level * stride] = rd_far;
          pending |= 1u << level;
        }
        stem_idx = stem_idx * 2u + (is_right ? 1u : 0u);
      } else {
        stem_idx = stem_idx * 2u;
      }
      ++level;
      dim = dim + 1 == K ? 0 : dim + 1;
    }
    cur = level;
    return stem_idx & ~(1u << level);
  }

  template <typename P>
  __device__ __forceinline__ bool backtrack(const TreeView<A>& tv, const A (&q)[K], const P& pol,
                                            A* __restrict__ slot, int stride) {
    while (cur > 0) {
      const int L = cur - 1;
      const int d = dim == 0 ? K - 1 : dim - 1;
      dim = d;
      const uint32_t bit = 1u << L;
      if (taken & bit) {
        put(off, d, slot[L * stride]);  // the restore frame of a far branch
        taken &= ~bit;
      } else if (pending & bit) {
        pending &= ~bit;
        const A frd = slot[L * stride];
        const A md = pol.max_dist();
        if (!(frd > md || (P::kPruneOnEqual && frd == md))) {
          const A pivot = __ldg(tv.stems + (stem_idx >> 1));
          const A old = sel(off, d);
          slot[L * stride] = old;
          taken |= bit;
          put(off, d, abs_val(sub_rn(sel(q, d), pivot)));
          rd = frd;
          stem_idx ^= 1u;
          level = cur;
          dim = d + 1 == K ? 0 : d + 1;
          return true;
        }
      }
      stem_idx >>= 1;
      cur = L;
    }
    return false;
  }

  __device__ __forceinline__ uint2 leaf_extents(const TreeView<A>& tv, uint32_t l) const {
    return __ldg(tv.extents + l);
  }
};

// Per-thread scalar backtracking, the reference's path for Donnelly<bh>
// stems (BLOCK_SIZE != 1) and for Mapped resolution over either stem order
// (kd_tree/orchestrator/mod.rs:214-345, 607-669; traits/stem_strategy.rs:
// 209-325): a Mapped tree's terminal stems end a descent at their leaf.  The reference's stack
// holds frames at strictly increasing levels, so the frame of the far child at
// level FL lives in slot FL of three shared-memory columns (its rd, the off
// value to put on its parent's axis, its stem index) with a bit in `pending`;
// its dimension is (FL - 1) % K, its minor level FL % bh and its leaf-index
// prefix the current path's at FL with the last bit flipped.  As in the
// reference, a descent keeps the popped frame's rd, pushes a far child when
// rd_far is not greater than max_dist() read when the descent began, and a pop
// resets only its own axis of `off`.
template <typename A, int K, typename M>
struct DonnellyWalk {
  A off[K];
  A rd;
  uint32_t stem, leaf, pending;
  int level;
  A* __restrict__ off_slot;         // column base: slot L at L * stride
  uint32_t* __restrict__ stem_slot;

  __device__ DonnellyWalk(A* offs, uint32_t* stems) : off_slot(offs), stem_slot(stems) {}

  __device__ __forceinline__ uint2 leaf_extents(const TreeView<A>& tv, uint32_t l) const {
    return __ldg(tv.extents + l);
  }

  __device__ __forceinline__ void init() {
#pragma unroll
    for (int d = 0; d < K; ++d) off[d] = A(0);
    rd = A(0);
    stem = leaf = pending = 0;
    level = 0;
  }

  template <typename P>
  __device__ __forceinline__ uint32_t descend(const TreeView<A>& tv, const A (&q)[K], const P& pol,
                                              bool, A* __restrict__ slot, int stride,
                                              TravStats& st) {
    const A INF = inf_of<A>();
    const A best = pol.max_dist();
    const int msl = tv.max_stem_level;
    if (!tv.bh && stem == 0) stem = 1;  // a fresh walk starts at the Eytzinger root
    int dim = level % K;
    uint32_t tl;
    while (level <= msl) {
      // a Mapped tree's terminal stem is a leaf (traverse_to_leaf,
      // orchestrator/mod.rs:624-631)
      if (terminal_leaf(tv, stem, tl)) return tl;
      ++st.stems;
      const A pivot = stem < tv.stem_count ? __ldg(tv.stems + stem) : INF;
      uint32_t l, r;
      stem_children(tv, stem, level, l, r);
      if (pivot < INF) {
        const A qd = sel(q, dim);
        const bool is_right = qd >= pivot;
        const A new_off = abs_val(sub_rn(qd, pivot));
        const A rd_far = M::template rect_k<A, K>(rd, off, dim, new_off);
        if (!(rd_far > best)) {
          const int fl = level + 1;
          slot[fl * stride] = rd_far;
          off_slot[fl * stride] = new_off;
          stem_slot[fl * stride] = is_right ? l : r;
          pending |= 1u << fl;
        }
        stem = is_right ? r : l;
        leaf = (leaf << 1) | (is_right ? 1u : 0u);
      } else {
        stem = l;
        leaf <<= 1;
      }
      ++level;
      dim = dim + 1 == K ? 0 : dim + 1;
    }
    if (tv.leaf_map && terminal_leaf(tv, stem, tl)) return tl;
    return leaf;
  }

  template <typename P>
  __device__ __forceinline__ bool backtrack(const TreeView<A>&, const A (&)[K], const P& pol,
                                            A* __restrict__ slot, int stride) {
    while (pending) {
      const int fl = 31 - __clz(pending);
      pending &= ~(1u << fl);
      const A frd = slot[fl * stride];
      const A md = pol.max_dist();
      if (frd > md || (P::kPruneOnEqual && frd == md)) continue;
      put(off, (fl - 1) % K, off_slot[fl * stride]);
      stem = stem_slot[fl * stride];
      leaf = (leaf >> (level - fl)) ^ 1u;
      level = fl;
      rd = frd;
      return true;
    }
    return false;
  }
};

// Per-thread periodic_backtracking_query (periodic.rs:455-619).  The
// reference's frames carry the far child's whole (lower, upper, off) state;
// here a frame is only its rd (slot[FL * stride], FL = the far child's level)
// and a bit in `frames`.  The rest is rebuilt when the frame is popped:
//  * the bound of axis d is the pivot of the deepest ancestor step that set
//    it (bit L of lo_set / hi_set: the step out of level L made lower /
//    upper of axis L % K equal to that stem's pivot), else 0 / the box size;
//  * off of axis d is periodic_interval_distance of those bounds once some
//    ancestor step split axis d (bit L of `split`), else 0.
// Both are exactly what the reference's step computed from the same inputs,
// so the rebuilt state equals the frame it replaces.
// STEMS == 0: Eytzinger stems, where an ancestor's index is the current
// index shifted right.  STEMS == 1: Donnelly<bh> stems or Mapped resolution
// (either stem order, terminal stems ending a descent), where the walk keeps
// the stem index of each level of its path in a column (path[L * stride])
// and the leaf index in `leaf`, one path bit per level; the traversal is the
// same (periodic.rs drives both stem orders through the StemStrategy trait).
// The cell state (lower bound, upper bound and interval offset of every
// axis) lives in 3K shared-memory columns of the thread (`bnd`: lower of axis
// d at d * pstride, upper at (K + d) * pstride, offset at (2K + d) * pstride),
// so it holds no registers while the warp scans leaves.
template <typename A, int K, typename M, int STEMS = 0>
struct PeriodicWalk {
  static constexpr uint32_t kDone = 0xffffffffu;
  A rd;
  uint32_t stem_idx, leaf;
  int level;
  uint32_t frames, split, lo_set, hi_set;
  bool at_leaf;
  uint32_t* __restrict__ path;  // Donnelly: this thread's column of path stem indices
  A* __restrict__ bnd;          // this thread's cell-bound columns
  int pstride;

  __device__ PeriodicWalk(uint32_t* p, A* bounds, int ps) : path(p), bnd(bounds), pstride(ps) {}

  __device__ __forceinline__ A lo(int d) const { return bnd[d * pstride]; }
  __device__ __forceinline__ A hi(int d) const { return bnd[(K + d) * pstride]; }
  __device__ __forceinline__ void set_lo(int d, A v) { bnd[d * pstride] = v; }
  __device__ __forceinline__ void set_hi(int d, A v) { bnd[(K + d) * pstride] = v; }
  __device__ __forceinline__ A off(int d) const { return bnd[(2 * K + d) * pstride]; }
  __device__ __forceinline__ void set_off(int d, A v) { bnd[(2 * K + d) * pstride] = v; }
  // the metric's rect_dist_after_update with axis `dim`'s offset replaced
  __device__ __forceinline__ A rect_after(int dim, A new_off) const {
    if constexpr (M::kAdditive) {
      return M::template rect<A>(rd, off(dim), new_off);
    } else {
      A o[K];
#pragma unroll
      for (int d = 0; d < K; ++d) o[d] = off(d);
      return M::template rect_k<A, K>(rd, o, dim, new_off);
    }
  }

  __device__ __forceinline__ static uint32_t axis_levels(int d) {
    uint32_t m = 0;
    for (int l = d; l < 32; l += K) m |= 1u << l;
    return m;
  }

  __device__ __forceinline__ void init(const A (&box)[K]) {
#pragma unroll
    for (int d = 0; d < K; ++d) {
      set_lo(d, A(0));
      set_hi(d, box[d]);
      set_off(d, A(0));
    }
    rd = A(0);
    stem_idx = STEMS ? 0u : 1u;
    leaf = 0;
    level = 0;
    frames = split = lo_set = hi_set = 0;
    at_leaf = false;
  }

  // Stem index of the path's node at level L <= P, where `parent` is the
  // node at level P.
  __device__ __forceinline__ uint32_t ancestor(uint32_t parent, int P, int L) const {
    if constexpr (STEMS) return path[L * pstride];
    else return parent >> (P - L);
  }

  // Pops the deepest pending frame (the reference's stack.pop()); false when
  // there is none.
  __device__ __forceinline__ bool pop(const TreeView<A>& tv, const A (&q)[K], const A (&box)[K],
                                      const A* __restrict__ slot, int stride) {
    if (!frames) return false;
    const int FL = 31 - __clz(frames);
    frames &= ~(1u << FL);
    const int P = FL - 1;
    const uint32_t parent = STEMS ? path[P * pstride] : stem_idx >> (level - P);
    const uint32_t below = (1u << P) - 1u;
    const int dP = P % K;
    A old_lo = A(0), old_hi = A(0);
#pragma unroll
    for (int d = 0; d < K; ++d) {
      const uint32_t am = axis_levels(d) & below;
      const uint32_t ml = lo_set & am, mh = hi_set & am;
      const A l = ml ? __ldg(tv.stems + ancestor(parent, P, 31 - __clz(ml))) : A(0);
      const A h = mh ? __ldg(tv.stems + ancestor(parent, P, 31 - __clz(mh))) : box[d];
      set_lo(d, l);
      set_hi(d, h);
      set_off(d, (split & am) ? periodic_interval_distance(q[d], l, h, box[d]) : A(0));
      if (d == dP) {
        old_lo = l;
        old_hi = h;
      }
    }
    const A pivot = __ldg(tv.stems + parent);
    const A qd = sel(q, dP);
    const bool is_right = qd >= pivot;
    const A minup = old_hi < pivot ? old_hi : pivot;
    const A maxlo = max_ref(old_lo, pivot);
    const A far_lo = is_right ? old_lo : maxlo;
    const A far_hi = is_right ? minup : old_hi;
    set_lo(dP, far_lo);
    set_hi(dP, far_hi);
    set_off(dP, periodic_interval_distance(qd, far_lo, far_hi, sel(box, dP)));
    rd = slot[FL * stride];
    split &= below;
    lo_set &= below;
    hi_set &= below;
    split |= 1u << P;
    if (!is_right && pivot > old_lo) lo_set |= 1u << P;   // far = right child: lower = maxlo
    if (is_right && !(old_hi < pivot)) hi_set |= 1u << P;  // far = left child: upper = minup
    if constexpr (STEMS) {
      uint32_t l, r;
      stem_children(tv, parent, P, l, r);
      stem_idx = is_right ? l : r;
      leaf = ((leaf >> (level - P)) << 1) | (is_right ? 0u : 1u);
    } else {
      stem_idx = parent * 2u + (is_right ? 0u : 1u);
    }
    level = FL;
    return true;
  }

  // The next leaf of the walk, or kDone.
  template <typename P>
  __device__ __forceinline__ uint32_t next(const TreeView<A>& tv, const A (&q)[K],
                                           const A (&box)[K], const P& pol, A* __restrict__ slot,
                                           int stride, TravStats& st) {
    if (at_leaf) {
      at_leaf = false;
      if (!pop(tv, q, box, slot, stride)) return kDone;
    }
    const A INF = inf_of<A>();
    const int msl = tv.max_stem_level;
    if (STEMS && !tv.bh && level == 0 && stem_idx == 0) stem_idx = 1;  // Eytzinger root
    int dim = level % K;
    for (;;) {
      uint32_t tl;
      if (STEMS && terminal_leaf(tv, stem_idx, tl)) {  // resolve_terminal_stem (periodic.rs:496-500)
        at_leaf = true;
        return tl;
      }
      if (level > msl) {
        at_leaf = true;
        if (STEMS && tv.leaf_map && terminal_leaf(tv, stem_idx, tl)) return tl;
        return STEMS ? leaf : (stem_idx & ~(1u << level));
      }
      ++st.stems;
      const A pivot = stem_idx < tv.stem_count ? __ldg(tv.stems + stem_idx) : INF;
      if constexpr (STEMS) path[level * pstride] = stem_idx;
      if (!(pivot < INF)) {
        if constexpr (STEMS) {
          uint32_t l, r;
          stem_children(tv, stem_idx, level, l, r);
          stem_idx = l;
          leaf <<= 1;
        } else {
          stem_idx *= 2u;
        }
        ++level;
        dim = dim + 1 == K ? 0 : dim + 1;
        continue;
      }
      const A old_lo = lo(dim), old_hi = hi(dim);
      const A qd = sel(q, dim), Ld = sel(box, dim);
      const bool is_right = qd >= pivot;
      const A minup = old_hi < pivot ? old_hi : pivot;
      const A maxlo = max_ref(old_lo, pivot);
      const A near_lo = is_right ? maxlo : old_lo;
      const A near_hi = is_right ? old_hi : minup;
      const A far_lo = is_right ? old_lo : maxlo;
      const A far_hi = is_right ? minup : old_hi;
      const A near_off = periodic_interval_distance(qd, near_lo, near_hi, Ld);
      const A far_off = periodic_interval_distance(qd, far_lo, far_hi, Ld);
      const A near_rd = rect_after(dim, near_off);
      const A far_rd = rect_after(dim, far_off);
      const A thr = pol.max_dist();
      const bool near_pruned = near_rd > thr || (P::kPruneOnEqual && near_rd == thr);
      const bool far_pruned = far_rd > thr || (P::kPruneOnEqual && far_rd == thr);
      if (!far_pruned) {
        slot[(level + 1) * stride] = far_rd;
        frames |= 1u << (level + 1);
      }
      if (near_pruned) {
        if (!pop(tv, q, box, slot, stride)) return kDone;
        dim = level % K;
        continue;
      }
      const uint32_t bit = 1u << level;
      split |= bit;
      if (is_right && pivot > old_lo) lo_set |= bit;
      if (!is_right && !(old_hi < pivot)) hi_set |= bit;
      set_lo(dim, near_lo);
      set_hi(dim, near_hi);
      set_off(dim, near_off);
      rd = near_rd;
      if constexpr (STEMS) {
        uint32_t l, r;
        stem_children(tv, stem_idx, level, l, r);
        stem_idx = is_right ? r : l;
        leaf = (leaf << 1) | (is_right ? 1u : 0u);
      } else {
        stem_idx = stem_idx * 2u + (is_right ? 1u : 0u);
      }
      ++level;
      dim = dim + 1 == K ? 0 : dim + 1;
    }
  }
};

// ---------------------------------------------------------------------------
// Thread policies
// ---------------------------------------------------------------------------
// Distance of a leaf point to the query (binds the query for the leaf walk).
template <typename A, int K, typename M>
struct CartesianQ {
  const A (&q)[K];
  __device__ __forceinline__ A operator()(const A (&c)[K]) const {
    return point_dist<M, A, K>(c, q);
  }
  // Both points of an f32 pair (v[d] = {axis d of point 0, of point 1}):
  // dist1 packed, the sum scalar in the order of point_dist.
  __device__ __forceinline__ void pair(const float2 (&v)[K], float& d0, float& d1) const {
    if constexpr (!M::kPacked) {
      float c0[K], c1[K];
#pragma unroll
      for (int d = 0; d < K; ++d) {
        c0[d] = v[d].x;
        c1[d] = v[d].y;
      }
      d0 = point_dist<M, float, K>(c0, q);
      d1 = point_dist<M, float, K>(c1, q);
      return;
    }
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int d = 0; d < K; ++d) {
      const F2 t = f2_sub(f2_pack(v[d].x, v[d].y), f2_pack(q[d], q[d]));
      F2 m;
      if constexpr (std::is_same<M, SqEuclidean>::value) m = f2_mul(t, t);
      else m = f2_abs(t);
      float m0, m1;
      f2_unpack(m, m0, m1);
      a0 = d ? __fadd_rn(a0, m0) : m0;
      a1 = d ? __fadd_rn(a1, m1) : m1;
    }
    d0 = a0;
    d1 = a1;
  }
};
template <typename A, int K, typename M>
struct TNearestOne {
  static constexpr bool kPruneOnEqual = true;
  A best;
  uint32_t item;
  __device__ TNearestOne() : best(inf_of<A>()), item(0) {}
  __device__ __forceinline__ void reset(A) { best = inf_of<A>(); item = 0; }
  __device__ __forceinline__ A max_dist() const { return best; }
  __device__ __forceinline__ bool unbounded_start() const { return true; }
  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint2 ex, const A (&q)[K]) {
    const CartesianQ<A, K, M> dist{q};
    return thread_for_each_point<A, K>(
        tv, ex, dist, [&](A d) { return d < best; },
        [&](A d, uint32_t it) {
          if (d < best) { best = d; item = it; }
        });
  }
};

// k smallest by (distance, arrival): the ThresholdVecResultCollection of
// results/result_collection.rs:136-215.  The list lives in shared memory, one
// column per thread (slot j of thread t at j * stride + t, so a warp touches
// 32 distinct banks whatever slot each thread is on).  While filling, hits are
// appended in arrival order; when the k-th arrives the list is sorted once,
// stably, by distance (std's small-slice sort is an insertion sort); after
// that a hit is inserted after equal distances, evicting the last.  A list
// that never fills stays in arrival order, which is ThresholdVec::into_vec;
// the sorted output sorts it at the end.
template <typename A, int K, typename M, bool kExclusive>
struct TNearestN {
  static constexpr bool kPruneOnEqual = kExclusive;
  // The list sits in shared-memory columns, entry j of thread t at j * stride + t.
  // For f32 an entry is one 8-byte (distance, item bits) pair, so moving an
  // entry is one 64-bit load and one 64-bit store; f64 keeps a distance column
  // and an item column.
  static constexpr bool kPacked = sizeof(A) == 4;
  using E = typename std::conditional<kPacked, float2, A>::type;
  E* __restrict__ le;
  uint32_t* __restrict__ li;  // f64 items
  int stride;
  int n, k;
  A radius, kth;
  // `lists` holds k * stride entries (k * stride * (sizeof(A) + 4) bytes)
  __device__ TNearestN(unsigned char* lists, int s, int k_, A r)
      : le(reinterpret_cast<E*>(lists) + threadIdx.x),
        li(reinterpret_cast<uint32_t*>(reinterpret_cast<A*>(lists) + size_t(k_) * s) +
           threadIdx.x),
        stride(s), n(0), k(k_), radius(r), kth(inf_of<A>()) {}
  __device__ __forceinline__ void reset(A r) { n = 0; radius = r; kth = inf_of<A>(); }
  __device__ __forceinline__ A max_dist() const { return (n == k && kth < radius) ? kth : radius; }
  __device__ __forceinline__ bool unbounded_start() const { return radius == inf_of<A>(); }

  __device__ __forceinline__ A dist_at(int j) const {
    if constexpr (kPacked) return le[j * stride].x;
    else return le[j * stride];
  }
  __device__ __forceinline__ uint32_t item_at(int j) const {
    if constexpr (kPacked) return __float_as_uint(le[j * stride].y);
    else return li[j * stride];
  }
  __device__ __forceinline__ void put(int j, A d, uint32_t it) {
    if constexpr (kPacked) {
      le[j * stride] = make_float2(d, __uint_as_float(it));
    } else {
      le[j * stride] = d;
      li[j * stride] = it;
    }
  }
  // Shifts the entries before position j that are above d one place up and
  // stores (d, it) in the gap: the stable insertion step (equal distances stay
  // ahead of the new entry).
  // Returns the distance now held at the starting position j: the entry that
  // moved into it, or d if d went there.
  __device__ __forceinline__ A insert_below(int j, A d, uint32_t it) {
    const int j0 = j;
    A top = d;
    if constexpr (kPacked) {
      // two entries read per step, so the shift waits on half as many
      // dependent shared-memory loads
      while (j > 1) {
        const float2 e1 = le[(j - 1) * stride];
        const float2 e2 = le[(j - 2) * stride];
        if (!(e1.x > d)) break;
        le[j * stride] = e1;
        if (j == j0) top = e1.x;
        if (!(e2.x > d)) {
          --j;
          break;
        }
        le[(j - 1) * stride] = e2;
        j -= 2;
      }
      if (j == 1) {
        const float2 e = le[0];
        if (e.x > d) {
          le[stride] = e;
          if (j == j0) top = e.x;
          j = 0;
        }
      }
    } else {
      while (j > 0 && le[(j - 1) * stride] > d) {
        le[j * stride] = le[(j - 1) * stride];
        li[j * stride] = li[(j - 1) * stride];
        if (j == j0) top = le[j * stride];
        --j;
      }
    }
    put(j, d, it);
    return top;
  }

  // stable insertion sort of the m held entries
  __device__ __forceinline__ void sort_held(int m) {
    for (int a = 1; a < m; ++a) insert_below(a, dist_at(a), item_at(a));
  }

  __device__ __forceinline__ void add(A d, uint32_t it) {
    if (n < k) {
      put(n, d, it);
      if (++n == k) {
        sort_held(k);
        kth = dist_at(k - 1);
      }
      return;
    }
    if (!(d < kth)) return;
    kth = insert_below(k - 1, d, it);
  }

  // The leaf filter of leaf_view_chunked/nearest_n_within/fallback.rs:37-95
  // (distance against max_dist() at leaf start, then the collector's own
  // test), in two passes per 32-point chunk: a convergent scan marks the
  // points that can enter the list (bound and, when the list starts full,
  // kth at leaf start), then the lanes insert their marked points in leaf
  // order together, each re-read from L1 and re-tested against the current
  // kth.  The add() calls are the sequential ones minus those add() would
  // reject, so the list is the same.
  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint2 ex, const A (&q)[K]) {
    // The mark "d within the leaf-start bound, and below kth when the list
    // started full" as one test d <= gate: strict comparisons become <= on
    // the next value down.
    A gate;
    if (n < k) {
      gate = kExclusive ? below(radius) : radius;
    } else if (kExclusive) {
      gate = below(kth < radius ? kth : radius);
    } else {
      gate = kth <= radius ? below(kth) : radius;
    }
    const CartesianQ<A, K, M> dist{q};
    const uint8_t* base = tv.arena + size_t(ex.x) * 8;
    const uint32_t len = ex.y;
    // every 128-byte line of the leaf's rows requested up front, so the scan's
    // one-row-per-step loads find them in L1
    if constexpr (RowLeaves<A, K>::value)
      for (uint32_t b = 0; b < len * row_bytes<A>(); b += 128u)
        asm volatile("prefetch.global.L1 [%0];" ::"l"(base + b));
    if constexpr (RowLeaves<A, K>::value && sizeof(A) == 4) {
      if (n == 0) {
        // A leaf reached with an empty list (every query's first): each point
        // that passes the gate is added, so one pass loads, measures and adds
        // the points in leaf order instead of marking them first.
        const float4* rows = reinterpret_cast<const float4*>(base);
        for (uint32_t p = 0; p < len; ++p) {
          const float4 v = __ldg(rows + p);
          const A c[K] = {v.x, v.y, v.z};
          const A d = dist(c);
          if (d <= gate) add(d, __float_as_uint(v.w));
        }
        return len;
      }
    }
    for (uint32_t c0 = 0; c0 < len; c0 += 32) {
      uint32_t mask = leaf_chunk_mask<A, K>(base, len, c0, dist, [&](A d) { return d <= gate; });
      if constexpr (RowLeaves<A, K>::value && sizeof(A) == 4) {
        // The next candidate's row is requested before the current one is
        // added, so its load overlaps the insertion (the kernel waits on load
        // latency more than on issue slots here).
        const float4* rows = reinterpret_cast<const float4*>(base);
        if (mask) {
          uint32_t p = c0 + uint32_t(__ffs(mask) - 1);
          mask &= mask - 1;
          float4 v = __ldg(rows + p);
          for (;;) {
            const bool more = mask != 0;
            float4 nv = v;
            if (more) {
              p = c0 + uint32_t(__ffs(mask) - 1);
              mask &= mask - 1;
              nv = __ldg(rows + p);
            }
            const A c[K] = {v.x, v.y, v.z};
            add(dist(c), __float_as_uint(v.w));
            if (!more) break;
            v = nv;
          }
        }
      } else {
        while (mask) {
          const uint32_t p = c0 + uint32_t(__ffs(mask) - 1);
          mask &= mask - 1;
          A c[K];
          uint32_t it;
          load_point<A, K>(base, len, p, c, it);
          add(dist(c), it);
        }
      }
    }
    return len;
  }

  __device__ __forceinline__ void write(uint64_t qi, A* __restrict__ out_d,
                                        uint32_t* __restrict__ out_i,
                                        uint32_t* __restrict__ out_c, bool arrival_order) {
    if (n < k && !arrival_order) sort_held(n);
    A* od = out_d + size_t(qi) * k;
    uint32_t* oi = out_i + size_t(qi) * k;
    for (int j = 0; j < k; ++j) {
      od[j] = j < n ? dist_at(j) : inf_of<A>();
      oi[j] = j < n ? item_at(j) : 0xffffffffu;
    }
    if (out_c) out_c[qi] = uint32_t(n);
  }
};

// best_n_within: the n smallest items among hits, by (item, arrival)
// (kd_tree/query/best_n_within.rs:88-196, leaf filter
// leaf_view_chunked/best_n_within/fallback.rs:40-104); list in shared memory
// kept sorted by item.
template <typename A, int K, typename M, bool kExclusive>
struct TBestN {
  static constexpr bool kPruneOnEqual = kExclusive;
  A* __restrict__ ld;
  uint32_t* __restrict__ li;
  int stride;
  int n, k;
  A radius;
  __device__ TBestN(A* d, uint32_t* i, int s, int k_, A r)
      : ld(d), li(i), stride(s), n(0), k(k_), radius(r) {}
  __device__ __forceinline__ void reset(A r) { n = 0; radius = r; }
  __device__ __forceinline__ A max_dist() const { return radius; }
  __device__ __forceinline__ bool unbounded_start() const { return false; }
  __device__ __forceinline__ void add(A d, uint32_t it) {
    int j;
    if (n < k) {
      j = n++;
    } else {
      if (!(it < li[(k - 1) * stride])) return;
      j = k - 1;
    }
    while (j > 0 && li[(j - 1) * stride] > it) {
      ld[j * stride] = ld[(j - 1) * stride];
      li[j * stride] = li[(j - 1) * stride];
      --j;
    }
    ld[j * stride] = d;
    li[j * stride] = it;
  }
  __device__ __forceinline__ uint32_t leaf(const TreeView<A>& tv, uint2 ex, const A (&q)[K]) {
    const bool full_at_entry = n == k;
    const uint32_t thr_item = full_at_entry ? li[(k - 1) * stride] : 0u;
    const CartesianQ<A, K, M> dist{q};
    return thread_for_each_point<A, K>(
        tv, ex, dist, [&](A d) { return kExclusive ? (d < radius) : (d <= radius); },
        [&](A d, uint32_t it) {
          if (!(kExclusive ? (d < radius) : (d <= radius))) return;
          if (full_at_entry && it >= thr_item) return;
          add(d, it);
        });
  }
  __device__ __forceinline__ void write(uint64_t qi, A* __restrict__ out_d,
                                        uint32_t* __restrict__ out_i,
                                        uint32_t* __restrict__ out_c) const {
    A* od = out_d + size_t(qi) * k;
    uint32_t* oi = out_i + size_t(qi) * k;
    for (int j = 0; j < k; ++j) {
      od[j] = j < n ? ld[j * stride] : inf_of<A>();
      oi[j] = j < n ? li[j * stride] : 0xffffffffu;
    }
    if (out_c) out_c[qi] = uint32_t(n);
  }
};

}  // namespace kgpu
