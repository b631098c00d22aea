// kiddo_oracle_capi.cpp — extern "C" surface of the CPU oracle for ctypes.
//
// TEST INFRASTRUCTURE ONLY (see kiddo_oracle.hpp).  Batch queries are spread
// over std::thread workers so the same code also serves as the timed CPU
// restatement of the reference path (a rayon par_iter over .execute() in
// benches/query.rs:36-52).
#include <atomic>
#include <cstdint>
#include <memory>
#include <thread>
#include <vector>

#include "kiddo_oracle.hpp"

using namespace kiddo_oracle;

namespace {

enum Family : int {
  FAM_NEAREST_ONE = 0,
  FAM_APPROX = 1,
  FAM_NEAREST_N = 2,       // nearest_n / nearest_n().within
  FAM_BEST_N_WITHIN = 3,
  FAM_PERIODIC_NEAREST_ONE = 4,
  FAM_PERIODIC_NEAREST_N = 5,
  FAM_WITHIN = 10,
  FAM_PERIODIC_WITHIN = 11,
};

struct TreeBase {
  int dtype;  // 0 f32, 1 f64
  int k;
  virtual ~TreeBase() = default;
};

template <typename A, int K>
struct TreeHolder : TreeBase {
  Tree<A, K> t;
};

struct RadiusResult {
  std::vector<uint64_t> offsets;
  std::vector<double> dists64;
  std::vector<float> dists32;
  std::vector<uint32_t> items;
  int dtype;
};

template <typename F>
void parallel_for(uint64_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 64) {
    for (uint64_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<uint64_t> next{0};
  const uint64_t chunk = 256;
  std::vector<std::thread> th;
  for (int w = 0; w < nthreads; ++w)
    th.emplace_back([&]() {
      for (;;) {
        uint64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        uint64_t e = std::min(n, b + chunk);
        for (uint64_t i = b; i < e; ++i) f(i);
      }
    });
  for (auto& x : th) x.join();
}

struct StatsAcc {
  std::atomic<uint64_t> stem{0}, leaf{0}, pts{0};
  void add(const Stats& s) {
    stem += s.stem_visits;
    leaf += s.leaf_visits;
    pts += s.points_scanned;
  }
};

template <typename A, int K, typename M>
int query_fixed_t(const Tree<A, K>& t, int family, const A* queries, uint64_t nq, uint32_t k,
                  A radius0, const A* radii, int exclusive, int sorted, const A* box, A* out_d,
                  uint32_t* out_i, uint32_t* out_c, int nthreads, uint64_t* stats3) {
  StatsAcc acc;
  const bool want_stats = stats3 != nullptr;
  parallel_for(nq, nthreads, [&](uint64_t qi) {
    Stats s;
    Stats* sp = want_stats ? &s : nullptr;
    const A* q = queries + qi * K;
    const A radius = radii ? radii[qi] : radius0;  // one radius per query, or one for all
    switch (family) {
      case FAM_NEAREST_ONE: {
        auto r = nearest_one<A, K, M>(t, q, sp);
        out_d[qi] = r.first; out_i[qi] = r.second;
        if (out_c) out_c[qi] = 1;
        break;
      }
      case FAM_APPROX: {
        auto r = approx_nearest_one<A, K, M>(t, q, sp);
        out_d[qi] = r.first; out_i[qi] = r.second;
        if (out_c) out_c[qi] = 1;
        break;
      }
      case FAM_PERIODIC_NEAREST_ONE: {
        if constexpr (M::kPeriodic) {
          auto r = periodic_nearest_one<A, K, M>(t, q, box, sp);
          out_d[qi] = r.first; out_i[qi] = r.second;
          if (out_c) out_c[qi] = 1;
        }
        break;
      }
      case FAM_NEAREST_N:
      case FAM_BEST_N_WITHIN:
      case FAM_PERIODIC_NEAREST_N: {
        std::vector<Hit<A>> h;
        if (family == FAM_NEAREST_N)
          h = nearest_n_within<A, K, M>(t, q, radius, k, exclusive, sorted, sp);
        else if (family == FAM_BEST_N_WITHIN)
          h = best_n_within<A, K, M>(t, q, radius, k, exclusive, sp);
        else if constexpr (M::kPeriodic)
          h = periodic_nearest<A, K, M>(t, q, box, radius, k, exclusive, sorted, sp);
        for (uint32_t j = 0; j < k; ++j) {
          if (j < h.size()) {
            out_d[qi * k + j] = h[j].dist;
            out_i[qi * k + j] = h[j].item;
          } else {
            out_d[qi * k + j] = inf_value<A>();
            out_i[qi * k + j] = 0xFFFFFFFFu;
          }
        }
        if (out_c) out_c[qi] = uint32_t(h.size());
        break;
      }
      default:
        break;
    }
    if (want_stats) acc.add(s);
  });
  if (want_stats) {
    stats3[0] = acc.stem;
    stats3[1] = acc.leaf;
    stats3[2] = acc.pts;
  }
  return 0;
}

template <typename A, int K, typename M>
RadiusResult* query_radius_t(const Tree<A, K>& t, int family, const A* queries, uint64_t nq,
                             A radius0, const A* radii, int exclusive, int sorted, const A* box,
                             int nthreads, uint64_t* stats3) {
  std::vector<std::vector<Hit<A>>> per(nq);
  StatsAcc acc;
  const bool want_stats = stats3 != nullptr;
  parallel_for(nq, nthreads, [&](uint64_t qi) {
    Stats s;
    Stats* sp = want_stats ? &s : nullptr;
    const A* q = queries + qi * K;
    const A radius = radii ? radii[qi] : radius0;
    if (family == FAM_WITHIN)
      per[qi] = within<A, K, M>(t, q, radius, exclusive, sorted, sp);
    else if constexpr (M::kPeriodic)
      per[qi] = periodic_nearest<A, K, M>(t, q, box, radius, 0, exclusive, sorted, sp);
    if (want_stats) acc.add(s);
  });
  auto* r = new RadiusResult();
  r->dtype = sizeof(A) == 8 ? 1 : 0;
  r->offsets.resize(nq + 1);
  uint64_t total = 0;
  for (uint64_t i = 0; i < nq; ++i) {
    r->offsets[i] = total;
    total += per[i].size();
  }
  r->offsets[nq] = total;
  r->items.resize(total);
  if (sizeof(A) == 8) r->dists64.resize(total); else r->dists32.resize(total);
  for (uint64_t i = 0; i < nq; ++i) {
    uint64_t o = r->offsets[i];
    for (size_t j = 0; j < per[i].size(); ++j) {
      r->items[o + j] = per[i][j].item;
      if (sizeof(A) == 8) r->dists64[o + j] = double(per[i][j].dist);
      else r->dists32[o + j] = float(per[i][j].dist);
    }
  }
  if (want_stats) {
    stats3[0] = acc.stem;
    stats3[1] = acc.leaf;
    stats3[2] = acc.pts;
  }
  return r;
}

template <typename F>
auto dispatch(int dtype, int k, F&& f) -> decltype(f(float(), std::integral_constant<int, 3>())) {
  using R = decltype(f(float(), std::integral_constant<int, 3>()));
#ifdef KOR_TIMING_BUILD
  // the timed CPU baseline needs 3-D trees only; fewer instantiations keep its
  // -O3 -march=native build short enough to run on the host being timed
  if (k == 3) {
    if (dtype == 0) return f(float(), std::integral_constant<int, 3>());
    if (dtype == 1) return f(double(), std::integral_constant<int, 3>());
  }
#else
  if (dtype == 0) {
    switch (k) {
      case 1: return f(float(), std::integral_constant<int, 1>());
      case 2: return f(float(), std::integral_constant<int, 2>());
      case 3: return f(float(), std::integral_constant<int, 3>());
      case 4: return f(float(), std::integral_constant<int, 4>());
    }
  } else if (dtype == 1) {
    switch (k) {
      case 1: return f(double(), std::integral_constant<int, 1>());
      case 2: return f(double(), std::integral_constant<int, 2>());
      case 3: return f(double(), std::integral_constant<int, 3>());
      case 4: return f(double(), std::integral_constant<int, 4>());
    }
  }
#endif
  return R();
}

}  // namespace

extern "C" {

// Build a tree with the restated soft construction.  `items` may be null, in
// which case item = source index (new_from_slice).  bh == 0: Eytzinger
// (ImmutableKdTree); bh > 0: Donnelly<bh>.
void* kor_build_ex(int dtype, int k, const void* pts, const uint32_t* items, uint64_t n,
                   uint32_t bh) {
  // Donnelly block heights the reference uses (3 for f64, 4 for f32 trees);
  // the core's bottom-row column min_idx - minor - 1 underflows below 3.
  if (bh != 0 && bh != 3 && bh != 4) return nullptr;
  return dispatch(dtype, k, [&](auto a, auto kk) -> void* {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    std::vector<uint32_t> gen;
    if (!items) {
      gen.resize(n);
      for (uint64_t i = 0; i < n; ++i) gen[i] = uint32_t(i);
      items = gen.data();
    }
    auto* h = new TreeHolder<A, K>();
    h->dtype = dtype;
    h->k = K;
    h->t = build<A, K>(static_cast<const A*>(pts), items, n, bh);
    return static_cast<TreeBase*>(h);
  });
}

void* kor_build(int dtype, int k, const void* pts, const uint32_t* items, uint64_t n) {
  return kor_build_ex(dtype, k, pts, items, n, 0);
}

// Wrap an externally produced layout (for example the one the product builder
// made) so the oracle's queries can run on exactly those bytes.
void* kor_from_layout_ex(int dtype, int k, const void* stems, uint64_t stems_len,
                         const uint8_t* bytes, uint64_t bytes_len, const uint64_t* extents,
                         uint64_t leaf_count, int32_t max_stem_level, uint64_t size,
                         uint64_t max_leaf_len, uint32_t bh) {
  return dispatch(dtype, k, [&](auto a, auto kk) -> void* {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    auto* h = new TreeHolder<A, K>();
    h->dtype = dtype;
    h->k = K;
    const A* s = static_cast<const A*>(stems);
    h->t.stems.assign(s, s + stems_len);
    h->t.leaf_bytes.assign(bytes, bytes + bytes_len);
    h->t.extents.assign(extents, extents + 2 * leaf_count);
    h->t.max_stem_level = max_stem_level;
    h->t.size = size;
    h->t.max_leaf_len = max_leaf_len;
    h->t.stem_strategy = bh ? 1 : 0;
    h->t.bh = bh;
    return static_cast<TreeBase*>(h);
  });
}

void* kor_from_layout(int dtype, int k, const void* stems, uint64_t stems_len,
                      const uint8_t* bytes, uint64_t bytes_len, const uint64_t* extents,
                      uint64_t leaf_count, int32_t max_stem_level, uint64_t size,
                      uint64_t max_leaf_len) {
  return kor_from_layout_ex(dtype, k, stems, stems_len, bytes, bytes_len, extents, leaf_count,
                            max_stem_level, size, max_leaf_len, 0);
}

// MutableKdTree-style bulk build: hard buckets and Mapped resolution
// (build_hard).  `kind` 0: the reference's construction; 1: an irregular
// Mapped tree of random leaf depths (build_irregular, Eytzinger stems), with
// `seed`.  nullptr for an unsplittable bucket or an unsupported shape.
void* kor_build_mapped(int dtype, int k, const void* pts, const uint32_t* items, uint64_t n,
                       uint32_t bh, int kind, uint64_t seed) {
  if (bh != 0 && bh != 3 && bh != 4) return nullptr;
  return dispatch(dtype, k, [&](auto a, auto kk) -> void* {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    std::vector<uint32_t> gen;
    if (!items) {
      gen.resize(n);
      for (uint64_t i = 0; i < n; ++i) gen[i] = uint32_t(i);
      items = gen.data();
    }
    auto* h = new TreeHolder<A, K>();
    h->dtype = dtype;
    h->k = K;
    if (kind == 1) {
      build_irregular<A, K>(h->t, static_cast<const A*>(pts), items, n, seed);
    } else if (!build_hard<A, K>(h->t, static_cast<const A*>(pts), items, n, bh)) {
      delete h;
      return nullptr;
    }
    return static_cast<TreeBase*>(h);
  });
}

// The Mapped resolution of a tree: out[0] = 1 if mapped, out[1] = map length,
// out[2] = min_stem_leaf_idx; kor_copy_leaf_map writes the map (leaf index or
// 2^64 - 1 = None per stem index from min_stem_leaf_idx on).
void kor_leaf_map_info(void* hp, uint64_t* out) {
  auto* b = static_cast<TreeBase*>(hp);
  dispatch(b->dtype, b->k, [&](auto a, auto kk) -> int {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    auto& t = static_cast<TreeHolder<A, K>*>(b)->t;
    out[0] = t.mapped ? 1 : 0;
    out[1] = t.leaf_map.size();
    out[2] = t.map_min;
    return 0;
  });
}

void kor_copy_leaf_map(void* hp, uint64_t* out) {
  auto* b = static_cast<TreeBase*>(hp);
  dispatch(b->dtype, b->k, [&](auto a, auto kk) -> int {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    auto& t = static_cast<TreeHolder<A, K>*>(b)->t;
    std::memcpy(out, t.leaf_map.data(), t.leaf_map.size() * 8);
    return 0;
  });
}

// Gives a tree made by kor_from_layout_ex a Mapped resolution.
void kor_set_leaf_map(void* hp, const uint64_t* map, uint64_t len, uint64_t min_stem_leaf_idx) {
  auto* b = static_cast<TreeBase*>(hp);
  dispatch(b->dtype, b->k, [&](auto a, auto kk) -> int {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    auto& t = static_cast<TreeHolder<A, K>*>(b)->t;
    t.mapped = true;
    t.leaf_map.assign(map, map + len);
    t.map_min = min_stem_leaf_idx;
    return 0;
  });
}

void kor_free(void* h) { delete static_cast<TreeBase*>(h); }

// KdTreeIter::next (src/kd_tree/iter.rs:64-90): leaf 0 to leaf_count - 1,
// each leaf's entries by position (leaf_point_item), which for VecOfArenas is
// the tile order of for_each_point.  Writes size items and size * K points.
void kor_iter(void* hp, uint32_t* items_out, void* points_out) {
  auto* b = static_cast<TreeBase*>(hp);
  dispatch(b->dtype, b->k, [&](auto a, auto kk) -> int {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    auto& t = static_cast<TreeHolder<A, K>*>(b)->t;
    A* pts = static_cast<A*>(points_out);
    uint64_t r = 0;
    for (size_t l = 0; l < t.leaf_count(); ++l)
      t.for_each_point(l, [&](const A (&c)[K], uint32_t item) {
        items_out[r] = item;
        for (int d = 0; d < K; ++d) pts[r * K + d] = c[d];
        ++r;
      });
    return 0;
  });
}

// layout[0..6] = stems_len, leaf_bytes_len, leaf_count, max_stem_level, size, max_leaf_len,
// block height (0: Eytzinger)
void kor_layout_info(void* hp, int64_t* info) {
  auto* b = static_cast<TreeBase*>(hp);
  dispatch(b->dtype, b->k, [&](auto a, auto kk) -> int {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    auto& t = static_cast<TreeHolder<A, K>*>(b)->t;
    info[0] = int64_t(t.stems.size());
    info[1] = int64_t(t.leaf_bytes.size());
    info[2] = int64_t(t.leaf_count());
    info[3] = t.max_stem_level;
    info[4] = int64_t(t.size);
    info[5] = int64_t(t.max_leaf_len);
    info[6] = int64_t(t.bh);
    return 0;
  });
}

void kor_copy_layout(void* hp, void* stems_out, uint8_t* bytes_out, uint64_t* extents_out) {
  auto* b = static_cast<TreeBase*>(hp);
  dispatch(b->dtype, b->k, [&](auto a, auto kk) -> int {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    auto& t = static_cast<TreeHolder<A, K>*>(b)->t;
    if (stems_out) std::memcpy(stems_out, t.stems.data(), t.stems.size() * sizeof(A));
    if (bytes_out) std::memcpy(bytes_out, t.leaf_bytes.data(), t.leaf_bytes.size());
    if (extents_out) std::memcpy(extents_out, t.extents.data(), t.extents.size() * 8);
    return 0;
  });
}

// metric: 0 SquaredEuclidean, 1 Manhattan, 2 Chebyshev, 3 / 4 Minkowski<3> /
// Minkowski<4>; every metric and stem order also periodic.  Outputs are dense [nq * k]
// (k = 1 for the nearest-one families); unused slots hold +inf / 0xFFFFFFFF.
// radii: one radius per query in the tree's dtype, or nullptr for `radius` on every query.
int kor_query_fixed_r(void* hp, int family, int metric, const void* queries, uint64_t nq,
                      uint32_t k, double radius, const void* radii, int exclusive, int sorted,
                      const void* box, void* out_d, uint32_t* out_i, uint32_t* out_c,
                      int nthreads, uint64_t* stats3) {
  auto* b = static_cast<TreeBase*>(hp);
  return dispatch(b->dtype, b->k, [&](auto a, auto kk) -> int {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    auto& t = static_cast<TreeHolder<A, K>*>(b)->t;
    auto run = [&](auto m) -> int {
      return query_fixed_t<A, K, decltype(m)>(
          t, family, static_cast<const A*>(queries), nq, k, A(radius),
          static_cast<const A*>(radii), exclusive, sorted, static_cast<const A*>(box),
          static_cast<A*>(out_d), out_i, out_c, nthreads, stats3);
    };
    if (metric == 0) return run(SqEuclidean());
#ifndef KOR_TIMING_BUILD
    if (metric == 1) return run(Manhattan());
    if (metric == 2) return run(Chebyshev());
    if (metric == 3) return run(Minkowski<3>());
    if (metric == 4) return run(Minkowski<4>());
#endif
    return -1;
  });
}

int kor_query_fixed(void* hp, int family, int metric, const void* queries, uint64_t nq,
                    uint32_t k, double radius, int exclusive, int sorted, const void* box,
                    void* out_d, uint32_t* out_i, uint32_t* out_c, int nthreads,
                    uint64_t* stats3) {
  return kor_query_fixed_r(hp, family, metric, queries, nq, k, radius, nullptr, exclusive,
                           sorted, box, out_d, out_i, out_c, nthreads, stats3);
}

void* kor_query_radius_r(void* hp, int family, int metric, const void* queries, uint64_t nq,
                         double radius, const void* radii, int exclusive, int sorted,
                         const void* box, int nthreads, uint64_t* stats3) {
  auto* b = static_cast<TreeBase*>(hp);
  return dispatch(b->dtype, b->k, [&](auto a, auto kk) -> void* {
    using A = decltype(a);
    constexpr int K = decltype(kk)::value;
    auto& t = static_cast<TreeHolder<A, K>*>(b)->t;
    auto run = [&](auto m) -> void* {
      return query_radius_t<A, K, decltype(m)>(
          t, family, static_cast<const A*>(queries), nq, A(radius),
          static_cast<const A*>(radii), exclusive, sorted, static_cast<const A*>(box), nthreads,
          stats3);
    };
    if (metric == 0) return run(SqEuclidean());
#ifndef KOR_TIMING_BUILD
    if (metric == 1) return run(Manhattan());
    if (metric == 2) return run(Chebyshev());
    if (metric == 3) return run(Minkowski<3>());
    if (metric == 4) return run(Minkowski<4>());
#endif
    return nullptr;
  });
}

void* kor_query_radius(void* hp, int family, int metric, const void* queries, uint64_t nq,
                       double radius, int exclusive, int sorted, const void* box, int nthreads,
                       uint64_t* stats3) {
  return kor_query_radius_r(hp, family, metric, queries, nq, radius, nullptr, exclusive, sorted,
                            box, nthreads, stats3);
}

// Test hook for the metric arithmetic (f64, K = 3): out[0] = dist(a, b),
// out[1] = rect_dist_after_update(rd, off, dim, new_off).
int kor_metric_f64x3(int metric, const double* a, const double* b, double rd, const double* off,
                     int dim, double new_off, double* out) {
  auto run = [&](auto m) {
    using M = decltype(m);
    out[0] = point_dist<M, double, 3>(a, b);
    out[1] = M::template rect_k<double, 3>(rd, off, dim, new_off);
    return 0;
  };
  if (metric == 0) return run(SqEuclidean());
  if (metric == 1) return run(Manhattan());
  if (metric == 2) return run(Chebyshev());
  if (metric == 3) return run(Minkowski<3>());
  if (metric == 4) return run(Minkowski<4>());
  return -1;
}

// Test hook for the Donnelly index math: walks `n` path bits from the root of
// a Donnelly<bh> stem tree.  out[0] = stem index after traverse() per bit;
// out[1], out[2] = the two children of the node reached by branch_relative()
// per bit (the two ways the reference moves a stem state).
void kor_donnelly_path(uint32_t bh, const uint8_t* bits, uint64_t n, uint32_t* out) {
  DonnellyCursor<3> a, b;
  a.bh = b.bh = bh;
  for (uint64_t i = 0; i < n; ++i) {
    a.traverse(bits[i] != 0);
    b.branch_relative(bits[i] != 0);
  }
  out[0] = a.stem_idx;
  b.children(out[1], out[2]);
}

uint64_t kor_radius_total(void* r) {
  auto* rr = static_cast<RadiusResult*>(r);
  return rr->offsets.back();
}

void kor_radius_copy(void* r, uint64_t* offsets, void* dists, uint32_t* items) {
  auto* rr = static_cast<RadiusResult*>(r);
  std::memcpy(offsets, rr->offsets.data(), rr->offsets.size() * 8);
  if (rr->dtype == 1) std::memcpy(dists, rr->dists64.data(), rr->dists64.size() * 8);
  else std::memcpy(dists, rr->dists32.data(), rr->dists32.size() * 4);
  std::memcpy(items, rr->items.data(), rr->items.size() * 4);
}

void kor_radius_free(void* r) { delete static_cast<RadiusResult*>(r); }

}  // extern "C"
