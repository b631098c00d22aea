// kgpu_forest.cu — batches over many trees in one launch, and CUDA-graph
// capture of query sequences.
//
// A forest is a device table of the member trees' views plus each tree's
// first global leaf number.  A forest query names the tree of every query
// (tree_of[qi]) and may give every query its own radius.  One persistent
// kernel answers the whole batch: warps take queries from a device work
// counter, so trees of very different sizes and queries with very different
// result counts do not leave SMs idle.  The radius fill takes a capacity and
// reports overflow in a device status word instead of reading the total back,
// so the whole count -> scan -> fill -> sort sequence can be captured in a
// CUDA graph and replayed.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kiddo_gpu.h"
#include "kgpu_device.cuh"
#include "kgpu_devbuf.h"
#include "kgpu_internal.h"
#include "kgpu_launch.h"
#include "kgpu_tree_impl.h"

struct kgpu_forest {
  kgpu::DeviceTree meta;       // dtype, dims; max_stem_level = the deepest member
  uint32_t n_trees = 0;
  void* views = nullptr;       // TreeView<A>[n_trees] on the device
  uint64_t* leaf_base = nullptr;
  uint64_t total_leaves = 0;
};

struct kgpu_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace kgpu {
namespace {

int cuda_err(cudaError_t e, const char* what) {
  return set_error(KGPU_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}


template <typename A>
void fill_views(const std::vector<kgpu_tree*>& trees, std::vector<uint8_t>& out) {
  out.resize(trees.size() * sizeof(TreeView<A>));
  for (size_t i = 0; i < trees.size(); ++i) {
    const DeviceTree& t = trees[i]->dt;
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
    std::memcpy(out.data() + i * sizeof(TreeView<A>), &v, sizeof(v));
  }
}

// Launch description of a forest query; the caller fills family-specific parts.
int forest_launch(kgpu_forest* f, const kgpu_query_desc* d, const void* queries,
                  const uint32_t* tree_of, const void* radii, uint64_t nq, QueryLaunch& q,
                  bool radius_family) {
  if (!f || !d) return set_error(KGPU_EINVAL, "NULL argument");
  // Validate against a tree-shaped stand-in carrying the forest's dtype/dims.
  kgpu_tree stand_in;
  stand_in.dt = f->meta;
  int st = check_query_desc(&stand_in, d, radius_family);
  if (st != KGPU_OK) return st;
  if (d->flags & KGPU_FLAG_HOST_BUFFERS)
    return set_error(KGPU_EINVAL, "forest queries take device pointers");
  if (nq && (!queries || !tree_of)) return set_error(KGPU_EINVAL, "queries or tree_of is NULL");
  q.family = d->family;
  q.metric = d->metric;
  q.k = (d->family == KGPU_NEAREST_ONE || d->family == KGPU_APPROX_NEAREST_ONE) ? 1
                                                                                : int(d->max_qty);
  q.radius = d->family == KGPU_NEAREST_N ? __builtin_inf() : d->radius;
  q.exclusive = d->exclusive != 0;
  q.sorted = rows_sorted(d);
  q.nq = nq;
  q.queries = queries;
  q.forest = f->views;
  q.tree_of = tree_of;
  q.n_trees = f->n_trees;
  q.leaf_base = f->leaf_base;
  q.total_leaves = f->total_leaves;
  q.radii = radii;
  apply_periodic(f->meta, d, q);
  q.engine = engine_of(d->flags);
  apply_tuning(d->tuning, q);
  return KGPU_OK;
}

// Work counter and optional leaf-bucketed order for one launch.
cudaError_t prepare(kgpu_forest* f, const kgpu_query_desc* d, QueryLaunch& q, DevBuf& work,
                    DevBuf& ord, DevBuf& scratch, cudaStream_t s) {
  cudaError_t e = work.alloc(sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(work.p, 0, sizeof(unsigned long long), s)) != cudaSuccess) return e;
  q.work = static_cast<unsigned long long*>(work.p);
  if (want_spatial_order(d->flags, q.nq, f->total_leaves)) {
    if ((e = ord.alloc(q.nq * 4, s)) != cudaSuccess) return e;
    if ((e = scratch.alloc(spatial_order_scratch_bytes(f->meta, q), s)) != cudaSuccess) return e;
    e = f->meta.dtype == KGPU_F64
            ? launch_spatial_order<double>(f->meta, q, static_cast<uint32_t*>(ord.p), scratch.p)
            : launch_spatial_order<float>(f->meta, q, static_cast<uint32_t*>(ord.p), scratch.p);
    if (e != cudaSuccess) return e;
    q.order = static_cast<uint32_t*>(ord.p);
  }
  return cudaSuccess;
}

}  // namespace
}  // namespace kgpu

using namespace kgpu;

extern "C" {

int32_t kgpu_forest_create(kgpu_tree* const* trees, uint32_t n_trees, void* stream,
                           kgpu_forest** out) {
  if (!out || (n_trees && !trees)) return set_error(KGPU_EINVAL, "NULL argument");
  *out = nullptr;
  if (n_trees == 0) return set_error(KGPU_EINVAL, "a forest needs at least one tree");
  std::vector<kgpu_tree*> ts(trees, trees + n_trees);
  int cur = -1;
  cudaGetDevice(&cur);
  for (auto* t : ts) {
    if (!t) return set_error(KGPU_EINVAL, "NULL tree in the forest");
    if (t->dt.dtype != ts[0]->dt.dtype || t->dt.dims != ts[0]->dt.dims)
      return set_error(KGPU_EINVAL, "forest trees must share dtype and dims");
    // one stem order per forest: the kernels walk Eytzinger stems, or
    // Donnelly stems of one block height
    if (t->dt.bh != ts[0]->dt.bh)
      return set_error(KGPU_EINVAL, "forest trees must share the stem order (and block height)");
    if ((t->dt.leaf_map != nullptr) != (ts[0]->dt.leaf_map != nullptr))
      return set_error(KGPU_EINVAL,
                       "forest trees must share the stem/leaf resolution (Mapped or arithmetic)");
    if (t->dt.device != cur) return set_error(KGPU_EINVAL, "forest trees must be on the current device");
  }
  auto* f = new (std::nothrow) kgpu_forest();
  if (!f) return set_error(KGPU_ENOMEM, "host allocation failed");
  f->n_trees = n_trees;
  f->meta.dtype = ts[0]->dt.dtype;
  f->meta.dims = ts[0]->dt.dims;
  f->meta.device = cur;
  f->meta.max_stem_level = -1;
  f->meta.size = 1;
  f->meta.bh = ts[0]->dt.bh;
  // routes the forest to the scalar walk; each query reads its own tree's map
  f->meta.leaf_map = ts[0]->dt.leaf_map;
  std::vector<uint64_t> base(n_trees);
  uint64_t total = 0;
  for (uint32_t i = 0; i < n_trees; ++i) {
    f->meta.max_stem_level = std::max(f->meta.max_stem_level, ts[i]->dt.max_stem_level);
    base[i] = total;
    total += std::max<uint32_t>(ts[i]->dt.leaf_count, 1u);
  }
  f->total_leaves = total;
  f->meta.leaf_count = uint32_t(std::min<uint64_t>(total, 0xffffffffull));
  std::vector<uint8_t> views;
  if (f->meta.dtype == KGPU_F64) fill_views<double>(ts, views);
  else fill_views<float>(ts, views);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if ((e = cudaMalloc(&f->views, views.size())) != cudaSuccess ||
      (e = cudaMalloc(reinterpret_cast<void**>(&f->leaf_base), base.size() * 8)) != cudaSuccess ||
      (e = cudaMemcpyAsync(f->views, views.data(), views.size(), cudaMemcpyHostToDevice, s)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(f->leaf_base, base.data(), base.size() * 8, cudaMemcpyHostToDevice,
                           s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    cudaFree(f->views);
    cudaFree(f->leaf_base);
    delete f;
    return cuda_err(e, "creating the forest");
  }
  *out = f;
  return KGPU_OK;
}

int32_t kgpu_forest_destroy(kgpu_forest* f) {
  if (!f) return KGPU_OK;
  cudaFree(f->views);
  cudaFree(f->leaf_base);
  delete f;
  return KGPU_OK;
}

int32_t kgpu_forest_query(kgpu_forest* f, const kgpu_query_desc* d, const void* queries,
                          const uint32_t* tree_of, const void* radii, uint64_t nq,
                          void* out_dists, uint32_t* out_items, uint32_t* out_counts,
                          void* stream) {
  QueryLaunch q;
  int st = forest_launch(f, d, queries, tree_of, radii, nq, q, false);
  if (st != KGPU_OK) return st;
  if (nq == 0) return KGPU_OK;
  if (!out_dists || !out_items) return set_error(KGPU_EINVAL, "NULL output buffer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  q.stream = s;
  q.out_d = out_dists;
  q.out_i = out_items;
  q.out_c = out_counts;
  DevBuf work, ord, scratch;
  cudaError_t e = prepare(f, d, q, work, ord, scratch, s);
  if (e != cudaSuccess) return cuda_err(e, "preparing the batch");
  e = f->meta.dtype == KGPU_F64 ? launch_fixed<double>(f->meta, q) : launch_fixed<float>(f->meta, q);
  if (e != cudaSuccess) return cuda_err(e, "launching the forest query");
  return KGPU_OK;
}

int32_t kgpu_forest_query_radius_count(kgpu_forest* f, const kgpu_query_desc* d,
                                       const void* queries, const uint32_t* tree_of,
                                       const void* radii, uint64_t nq, uint64_t* offsets,
                                       void* stream) {
  QueryLaunch q;
  int st = forest_launch(f, d, queries, tree_of, radii, nq, q, true);
  if (st != KGPU_OK) return st;
  if (!offsets) return set_error(KGPU_EINVAL, "offsets is NULL");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  q.stream = s;
  DevBuf work, ord, scratch, tmp;
  cudaError_t e;
  if ((e = tmp.alloc(scan_tmp_bytes(nq), s)) != cudaSuccess)
    return set_error(KGPU_ENOMEM, "device allocation failed");
  if (nq) {
    if ((e = prepare(f, d, q, work, ord, scratch, s)) != cudaSuccess)
      return cuda_err(e, "preparing the batch");
    e = f->meta.dtype == KGPU_F64 ? launch_within_count<double>(f->meta, q, offsets)
                                  : launch_within_count<float>(f->meta, q, offsets);
    if (e != cudaSuccess) return cuda_err(e, "launching the counting pass");
  }
  e = launch_exclusive_scan(offsets, offsets, nq, tmp.p, s);
  if (e != cudaSuccess) return cuda_err(e, "launching the scan");
  return KGPU_OK;
}

int32_t kgpu_forest_query_radius_fill(kgpu_forest* f, const kgpu_query_desc* d,
                                      const void* queries, const uint32_t* tree_of,
                                      const void* radii, uint64_t nq, const uint64_t* offsets,
                                      uint64_t capacity, void* out_dists, uint32_t* out_items,
                                      int32_t* status, void* stream) {
  QueryLaunch q;
  int st = forest_launch(f, d, queries, tree_of, radii, nq, q, true);
  if (st != KGPU_OK) return st;
  if (!offsets) return set_error(KGPU_EINVAL, "offsets is NULL");
  if (nq == 0 || capacity == 0) return KGPU_OK;
  if (!out_dists || !out_items) return set_error(KGPU_EINVAL, "NULL output buffer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  q.stream = s;
  q.out_d = out_dists;
  q.out_i = out_items;
  q.capacity = capacity;
  q.status = status;
  q.sorted = d->family == KGPU_WITHIN && d->sorted != 0;
  DevBuf work, ord, scratch, sd, si;
  cudaError_t e = prepare(f, d, q, work, ord, scratch, s);
  if (e != cudaSuccess) return cuda_err(e, "preparing the batch");
  e = f->meta.dtype == KGPU_F64 ? launch_within_fill<double>(f->meta, q, offsets)
                                : launch_within_fill<float>(f->meta, q, offsets);
  if (e != cudaSuccess) return cuda_err(e, "launching the fill pass");
  if (q.sorted) {
    const size_t sa = f->meta.dtype == KGPU_F64 ? 8 : 4;
    if ((e = sd.alloc(capacity * sa, s)) != cudaSuccess || (e = si.alloc(capacity * 4, s)) != cudaSuccess)
      return set_error(KGPU_ENOMEM, "device allocation failed");
    e = f->meta.dtype == KGPU_F64
            ? launch_seg_sort<double>(offsets, nq, capacity, static_cast<double*>(out_dists),
                                      out_items, static_cast<double*>(sd.p),
                                      static_cast<uint32_t*>(si.p), s)
            : launch_seg_sort<float>(offsets, nq, capacity, static_cast<float*>(out_dists),
                                     out_items, static_cast<float*>(sd.p),
                                     static_cast<uint32_t*>(si.p), s);
    if (e != cudaSuccess) return cuda_err(e, "launching the segmented sort");
  }
  return KGPU_OK;
}

// ---- CUDA graphs ------------------------------------------------------------
int32_t kgpu_graph_begin(void* stream) {
  if (!stream) return set_error(KGPU_EINVAL, "capture needs a stream other than the legacy default");
  cudaError_t e = cudaStreamBeginCapture(static_cast<cudaStream_t>(stream),
                                         cudaStreamCaptureModeRelaxed);
  return e == cudaSuccess ? KGPU_OK : cuda_err(e, "cudaStreamBeginCapture");
}

int32_t kgpu_graph_end(void* stream, kgpu_graph** out) {
  if (!stream || !out) return set_error(KGPU_EINVAL, "NULL argument");
  *out = nullptr;
  auto* g = new (std::nothrow) kgpu_graph();
  if (!g) return set_error(KGPU_ENOMEM, "host allocation failed");
  cudaError_t e = cudaStreamEndCapture(static_cast<cudaStream_t>(stream), &g->graph);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) {
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return cuda_err(e, "ending the capture");
  }
  *out = g;
  return KGPU_OK;
}

int32_t kgpu_graph_launch(kgpu_graph* g, void* stream) {
  if (!g) return set_error(KGPU_EINVAL, "NULL graph");
  cudaError_t e = cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? KGPU_OK : cuda_err(e, "cudaGraphLaunch");
}

int32_t kgpu_graph_destroy(kgpu_graph* g) {
  if (!g) return KGPU_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return KGPU_OK;
}

}  // extern "C"
