// kgpu_api.cu — the extern "C" entry points declared in include/kiddo_gpu.h.
//
// Validation, upload of the reference layout, host staging, and the
// count -> scan -> fill -> sort pipeline of the radius families.  Every entry
// point returns a status; no C++ exception or CUDA error escapes the ABI.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/kiddo_gpu.h"
#include "kgpu_devbuf.h"
#include "kgpu_internal.h"
#include "kgpu_launch.h"
#include "kgpu_tree_impl.h"

namespace kgpu {

std::atomic<uint64_t> g_launches{0};

namespace {
thread_local std::string t_last_error;
}

int set_error(int status, const std::string& msg) {
  t_last_error = msg;
  return status;
}

static int cuda_fail(cudaError_t e, const char* what) {
  return set_error(KGPU_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  static std::mutex mu;
  static std::vector<int> cache;
  std::lock_guard<std::mutex> g(mu);
  if (dev >= int(cache.size())) cache.resize(dev + 1, 0);
  if (cache[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cache[dev] = n > 0 ? n : 1;
  }
  return cache[dev];
}

namespace {

size_t leaf_encoded_bytes(uint64_t len, int K, size_t sa) {
  size_t total = 0;
  while (len) {
    uint64_t w = len >= 32 ? 32 : len >= 8 ? 8 : len >= 4 ? 4 : len >= 2 ? 2 : 1;
    total += size_t(w) * (K * sa + 4);
    len -= w;
  }
  return total;
}

}  // namespace
}  // namespace kgpu

namespace kgpu {

uint64_t current_context_id() {
  // cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points, so
  // the library needs no link-time dependency on the driver library
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult r;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &r) ==
            cudaSuccess && r == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &r) ==
            cudaSuccess && r == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

namespace {
// One stream-ordered pool per device, private to the library: its release
// threshold is at its maximum, so freed scratch stays cached across stream
// synchronizations instead of going back to the driver at each one (and being
// mapped again, milliseconds later, by the next call).  Being the library's
// own, the setting leaves the device's default pool (and every other
// cudaMallocAsync user in the process) as it was.  A pool belongs to a
// context: after cudaDeviceReset the next call makes a new one.
struct ScratchPool {
  uint64_t ctx_id = 0;
  cudaMemPool_t pool = nullptr;
};
constexpr int kPoolDevices = 64;
std::mutex g_pool_mu;
ScratchPool g_pools[kPoolDevices];
}  // namespace

cudaError_t library_pool(int dev, cudaMemPool_t* out) {
  if (dev < 0 || dev >= kPoolDevices) return cudaErrorInvalidDevice;
  const uint64_t ctx = current_context_id();
  std::lock_guard<std::mutex> g(g_pool_mu);
  ScratchPool& sp = g_pools[dev];
  if (!sp.pool || sp.ctx_id != ctx) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = ~uint64_t(0);
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return e;
    }
    sp.pool = pool;
    sp.ctx_id = ctx;
  }
  *out = sp.pool;
  return cudaSuccess;
}

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool = nullptr;
  if ((e = library_pool(dev, &pool)) != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

void release_tree_arrays(DeviceTree& dt) {
  cudaFree(dt.leaf_map);
  dt.leaf_map = nullptr;
  cudaFree(dt.iter_points);
  cudaFree(dt.sorted_items);
  cudaFree(dt.sorted_ranks);
  dt.iter_points = nullptr;
  dt.sorted_items = nullptr;
  dt.sorted_ranks = nullptr;
  dt.items_distinct = -1;
  if (dt.pooled) {
    // the arrays came from the device's stream-ordered pool: wait for every
    // stream, as cudaFree would, then return them to the pool
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dt.device) cudaSetDevice(dt.device);
    cudaDeviceSynchronize();
    if (dt.stems) cudaFreeAsync(dt.stems, nullptr);
    if (dt.arena) cudaFreeAsync(dt.arena, nullptr);
    if (dt.extents) cudaFreeAsync(dt.extents, nullptr);
    if (dt.src_extents) cudaFreeAsync(dt.src_extents, nullptr);
    cudaStreamSynchronize(nullptr);
    if (cur != dt.device) cudaSetDevice(cur);
  } else {
    cudaFree(dt.stems);
    cudaFree(dt.arena);
    cudaFree(dt.extents);
    cudaFree(dt.src_extents);
  }
  dt.stems = nullptr;
  dt.arena = nullptr;
  dt.extents = nullptr;
  dt.src_extents = nullptr;
}

}  // namespace kgpu

using namespace kgpu;

extern "C" {

const char* kgpu_last_error(void) { return t_last_error.c_str(); }

const char* kgpu_status_string(int32_t s) {
  switch (s) {
    case KGPU_OK: return "ok";
    case KGPU_EINVAL: return "invalid argument";
    case KGPU_EUNSUPPORTED: return "unsupported layout or option";
    case KGPU_ENOMEM: return "out of memory";
    case KGPU_ECUDA: return "CUDA error";
    case KGPU_ETIMEDOUT: return "device wait timed out";
    case KGPU_EOVERFLOW: return "capacity overflow";
    case KGPU_ENOTREADY: return "not ready";
  }
  return "unknown status";
}

uint32_t kgpu_abi_version(void) { return KGPU_ABI_VERSION; }

uint64_t kgpu_launch_count(void) { return g_launches.load(); }

namespace {
// The library's pool on `device` if one was made in the device's current
// context (nullptr otherwise), with that device current until `restore`.
struct PoolOnDevice {
  int prev = -1;
  cudaMemPool_t pool = nullptr;
  cudaError_t err = cudaSuccess;
  explicit PoolOnDevice(int device) {
    if ((err = cudaGetDevice(&prev)) != cudaSuccess) return;
    if (prev != device && (err = cudaSetDevice(device)) != cudaSuccess) return;
    const uint64_t ctx = current_context_id();
    std::lock_guard<std::mutex> g(g_pool_mu);
    if (g_pools[device].ctx_id == ctx) pool = g_pools[device].pool;
  }
  ~PoolOnDevice() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};
}  // namespace

int32_t kgpu_scratch_stats(int32_t device, uint64_t out[3]) {
  if (!out) return set_error(KGPU_EINVAL, "out is NULL");
  out[0] = out[1] = out[2] = 0;
  if (device < 0 || device >= kPoolDevices) return set_error(KGPU_EINVAL, "bad device index");
  PoolOnDevice pd(device);
  if (pd.err != cudaSuccess) return cuda_fail(pd.err, "selecting the device");
  if (!pd.pool) return KGPU_OK;
  const cudaMemPoolAttr attrs[3] = {cudaMemPoolAttrUsedMemCurrent, cudaMemPoolAttrUsedMemHigh,
                                    cudaMemPoolAttrReservedMemCurrent};
  for (int i = 0; i < 3; ++i) {
    cudaError_t e = cudaMemPoolGetAttribute(pd.pool, attrs[i], &out[i]);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolGetAttribute");
  }
  return KGPU_OK;
}

int32_t kgpu_scratch_trim(int32_t device) {
  if (device < 0 || device >= kPoolDevices) return set_error(KGPU_EINVAL, "bad device index");
  PoolOnDevice pd(device);
  if (pd.err != cudaSuccess) return cuda_fail(pd.err, "selecting the device");
  if (!pd.pool) return KGPU_OK;
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemPoolTrimTo(pd.pool, 0);
  uint64_t zero = 0;  // the high-water mark restarts from the bytes in use
  if (e == cudaSuccess) e = cudaMemPoolSetAttribute(pd.pool, cudaMemPoolAttrUsedMemHigh, &zero);
  return e == cudaSuccess ? KGPU_OK : cuda_fail(e, "trimming the scratch pool");
}

// ---- host construction ----------------------------------------------------
int32_t kgpu_layout_build(int32_t dtype, uint32_t dims, const void* points, const uint32_t* items,
                          uint64_t n, int32_t nthreads, kgpu_layout** out) {
  return kgpu_layout_build_stems(dtype, dims, points, items, n, KGPU_STEM_EYTZINGER, 0, nthreads,
                                 out);
}

int32_t kgpu_layout_build_stems(int32_t dtype, uint32_t dims, const void* points,
                                const uint32_t* items, uint64_t n, int32_t stem_strategy,
                                uint32_t block_height, int32_t nthreads, kgpu_layout** out) {
  if (!out) return set_error(KGPU_EINVAL, "out is NULL");
  *out = nullptr;
  if (stem_strategy == KGPU_STEM_EYTZINGER) {
    block_height = 0;
  } else if (stem_strategy != KGPU_STEM_DONNELLY) {
    return set_error(KGPU_EINVAL, "unknown stem strategy");
  } else if (block_height != 3 && block_height != 4) {
    return set_error(KGPU_EUNSUPPORTED, "Donnelly block height must be 3 or 4");
  }
  auto* lay = new (std::nothrow) kgpu_layout();
  if (!lay) return set_error(KGPU_ENOMEM, "host allocation failed");
  int st = build_layout_any(lay->L, dtype, int(dims), points, items, n, nthreads, block_height);
  if (st != KGPU_OK) {
    delete lay;
    return st;
  }
  *out = lay;
  return KGPU_OK;
}

int32_t kgpu_layout_describe(const kgpu_layout* lay, kgpu_tree_desc* d) {
  if (!lay || !d) return set_error(KGPU_EINVAL, "NULL argument");
  const Layout& L = lay->L;
  std::memset(d, 0, sizeof(*d));
  d->abi_version = KGPU_ABI_VERSION;
  d->dtype = L.dtype;
  d->dims = uint32_t(L.dims);
  d->item_size = 4;
  d->bucket_size = 32;
  d->stem_strategy = L.block_height ? KGPU_STEM_DONNELLY : KGPU_STEM_EYTZINGER;
  d->block_height = L.block_height;
  d->resolution = KGPU_RES_ARITHMETIC;
  const size_t sa = L.dtype == KGPU_F64 ? 8 : 4;
  d->stems = L.stems_bytes.empty() ? nullptr : L.stems_bytes.data();
  d->stem_count = L.stems_bytes.size() / sa;
  d->leaf_bytes = L.leaf_bytes.empty() ? nullptr : L.leaf_bytes.data();
  d->leaf_bytes_len = L.leaf_bytes.size();
  d->leaf_extents = L.extents.empty() ? nullptr : L.extents.data();
  d->leaf_count = L.extents.size() / 2;
  d->max_stem_level = L.max_stem_level;
  d->size = L.size;
  d->max_leaf_len = L.max_leaf_len;
  return KGPU_OK;
}

int32_t kgpu_layout_free(kgpu_layout* lay) {
  delete lay;
  return KGPU_OK;
}

// ---- device trees -----------------------------------------------------------
}  // extern "C"

namespace kgpu {
namespace {

// The stem index of a child in the tree's stem order (host side).
uint32_t host_child(uint32_t bh, uint32_t stem, int level, bool right) {
  if (!bh) return stem * 2u + (right ? 1u : 0u);
  const uint32_t minor = uint32_t(level) % bh;
  const uint32_t mask = (1u << bh) - 1u, min_idx = stem & mask, base = (stem & ~mask) + 1u;
  const uint32_t l = minor + 1u == bh ? (base + ((min_idx - minor - 1u) << 1)) << bh
                                      : base + (min_idx << 1);
  return right ? (minor + 1u == bh ? l + (1u << bh) : l + 1u) : l;
}

// Checks a Mapped resolution against its stems: every walk from the root ends
// at a terminal stem (resolve_terminal_stem) naming a leaf, at the latest just
// past max_stem_level, where the reference would otherwise panic
// (stem_leaf_resolution.rs:176-200).  A stem without a split continues to its
// left child only (traverse(false)).
bool mapped_walks_end_in_leaves(const kgpu_tree_desc* d, const std::vector<uint32_t>& map,
                                uint64_t map_min, uint32_t bh, uint32_t stem, int level) {
  const uint64_t mi = uint64_t(stem) - map_min;
  if (stem >= map_min && mi < map.size() && map[mi] != 0xffffffffu) return true;
  if (level > d->max_stem_level) return false;
  double pivot = __builtin_inf();
  if (stem < d->stem_count)
    pivot = d->dtype == KGPU_F64 ? static_cast<const double*>(d->stems)[stem]
                                 : double(static_cast<const float*>(d->stems)[stem]);
  if (!mapped_walks_end_in_leaves(d, map, map_min, bh, host_child(bh, stem, level, false),
                                  level + 1))
    return false;
  return !(pivot < __builtin_inf()) ||
         mapped_walks_end_in_leaves(d, map, map_min, bh, host_child(bh, stem, level, true),
                                    level + 1);
}

int create_tree(const kgpu_tree_desc* d, const kgpu_leaf_map* m, void* stream,
                kgpu_tree** out) {
  if (!d || !out) return set_error(KGPU_EINVAL, "NULL argument");
  *out = nullptr;
  if (d->abi_version != KGPU_ABI_VERSION) return set_error(KGPU_EINVAL, "abi_version mismatch");
  if (d->dtype != KGPU_F32 && d->dtype != KGPU_F64)
    return set_error(KGPU_EINVAL, "dtype must be KGPU_F32 or KGPU_F64");
  if (d->dims < 1 || d->dims > uint32_t(kMaxDims))
    return set_error(KGPU_EUNSUPPORTED, "dims must be 1..4");
  if (d->item_size != 4) return set_error(KGPU_EUNSUPPORTED, "only u32 items (ImmutableKdTree)");
  if (d->bucket_size != 32) return set_error(KGPU_EUNSUPPORTED, "only bucket size 32");
  const bool donnelly = d->stem_strategy == KGPU_STEM_DONNELLY;
  if (d->stem_strategy != KGPU_STEM_EYTZINGER && !donnelly)
    return set_error(KGPU_EINVAL, "unknown stem strategy");
  if (donnelly && d->block_height != 3 && d->block_height != 4)
    return set_error(KGPU_EUNSUPPORTED, "Donnelly block height must be 3 or 4");
  const bool mapped = m != nullptr;
  if (mapped ? d->resolution != KGPU_RES_MAPPED
             : (d->resolution != KGPU_RES_ARITHMETIC && d->resolution != KGPU_RES_PRISTINE))
    return set_error(KGPU_EINVAL,
                     mapped ? "a leaf map comes with KGPU_RES_MAPPED"
                            : "Mapped resolution needs its leaf map (kgpu_tree_create_mapped)");
  if (d->max_stem_level < -1 || d->max_stem_level > kMaxStemLevel)
    return set_error(KGPU_EUNSUPPORTED, "max_stem_level must be -1..30");
  const size_t sa = d->dtype == KGPU_F64 ? 8 : 4;
  const int K = int(d->dims);
  std::vector<uint32_t> lmap;
  if (mapped) {
    // the leaf map, as u32 leaf indices (0xffffffff: not terminal)
    if (m->len && !m->leaf_idx_map) return set_error(KGPU_EINVAL, "leaf_idx_map is NULL");
    if (m->len > 0xffffffffull || m->min_stem_leaf_idx > 0xffffffffull)
      return set_error(KGPU_EOVERFLOW, "leaf map beyond 32-bit stem indices");
    if (d->stem_count > 0xFFFFFFFFull)
      return set_error(KGPU_EOVERFLOW, "stem indices beyond 32 bits");
    if (d->max_stem_level >= 0 && !d->stems) return set_error(KGPU_EINVAL, "stems is NULL");
    try {
      lmap.resize(m->len);
    } catch (const std::bad_alloc&) {
      return set_error(KGPU_ENOMEM, "host allocation failed");
    }
    for (uint64_t i = 0; i < m->len; ++i) {
      const uint64_t v = m->leaf_idx_map[i];
      if (v == ~uint64_t(0)) {
        lmap[i] = 0xffffffffu;
      } else if (v >= d->leaf_count) {
        return set_error(KGPU_EINVAL, "leaf map names a leaf beyond leaf_count");
      } else {
        lmap[i] = uint32_t(v);
      }
    }
    if (d->size && !mapped_walks_end_in_leaves(d, lmap, m->min_stem_leaf_idx,
                                               donnelly ? d->block_height : 0, donnelly ? 0u : 1u,
                                               0))
      return set_error(KGPU_EINVAL, "a walk of the Mapped tree reaches no leaf");
  } else if (!donnelly) {
    const uint64_t expect_leaves =
        d->max_stem_level >= 0 ? (uint64_t(1) << (d->max_stem_level + 1)) : (d->size ? 1 : 0);
    if (d->leaf_count != expect_leaves)
      return set_error(KGPU_EINVAL,
                       "leaf_count does not match max_stem_level (arithmetic layout)");
    if (d->max_stem_level >= 0 && d->stem_count < (uint64_t(1) << (d->max_stem_level + 1)))
      return set_error(KGPU_EINVAL, "stem array shorter than 2^(max_stem_level+1)");
  } else if (d->max_stem_level >= 0) {
    // Donnelly: stems_depth = max_stem_level + 1 is a multiple of bh, the
    // first (padding) levels carry no split, and the 2^o leaves hang below
    // the o levels that do (construction.rs:431-446); stem loads are
    // bounds-checked against stem_count on the device.
    const uint32_t depth = uint32_t(d->max_stem_level + 1);
    if (depth % d->block_height)
      return set_error(KGPU_EINVAL, "Donnelly stem depth is not a multiple of the block height");
    uint32_t o = 0;
    while (o < 63 && (uint64_t(1) << o) < d->leaf_count) ++o;
    if (d->leaf_count == 0 || (uint64_t(1) << o) != d->leaf_count || o > depth ||
        depth - o >= d->block_height)
      return set_error(KGPU_EINVAL, "leaf_count does not match a Donnelly arithmetic layout");
    if (d->stem_count > 0xFFFFFFFFull)
      return set_error(KGPU_EOVERFLOW, "Donnelly stem indices beyond 32 bits");
    // The padding levels (the first depth - o, walked to the left) must carry
    // no split, so that the path bits of every leaf stay below leaf_count.
    const uint32_t bh = d->block_height;
    uint32_t stem = 0, minor = 0;
    for (uint32_t lvl = 0; lvl < depth - o; ++lvl) {
      if (stem < d->stem_count) {
        double v;
        if (d->dtype == KGPU_F64) v = static_cast<const double*>(d->stems)[stem];
        else v = double(static_cast<const float*>(d->stems)[stem]);
        if (v < __builtin_inf())
          return set_error(KGPU_EINVAL, "a Donnelly padding level holds a split");
      }
      const uint32_t mask = (1u << bh) - 1u, min_idx = stem & mask, base = (stem & ~mask) + 1u;
      stem = minor + 1u == bh ? (base + ((min_idx - minor - 1u) << 1)) << bh
                              : base + (min_idx << 1);
      minor = minor + 1u == bh ? 0u : minor + 1u;
    }
  } else if (d->leaf_count != (d->size ? 1u : 0u)) {
    return set_error(KGPU_EINVAL, "leaf_count does not match a tree without stems");
  }
  if (d->leaf_count && (!d->leaf_extents || !d->leaf_bytes))
    return set_error(KGPU_EINVAL, "leaf arrays are NULL");
  if (d->max_stem_level >= 0 && !d->stems) return set_error(KGPU_EINVAL, "stems is NULL");
  if (d->leaf_bytes_len / 8 >= (uint64_t(1) << 32))
    return set_error(KGPU_EOVERFLOW, "leaf arena larger than 32 GiB");
  // extents -> (offset / 8, len), validated against the arena
  std::vector<uint32_t> ex;
  try {
    ex.resize(2 * d->leaf_count);
  } catch (const std::bad_alloc&) {
    return set_error(KGPU_ENOMEM, "host allocation failed");
  }
  uint64_t total = 0;
  for (uint64_t l = 0; l < d->leaf_count; ++l) {
    const uint64_t off = d->leaf_extents[2 * l], len = d->leaf_extents[2 * l + 1];
    if (off % 8) return set_error(KGPU_EINVAL, "leaf offset not 8-byte aligned");
    // f32 3-D leaves are 16 bytes per point, so the reference's offsets are
    // multiples of 16; the device reads them as aligned 16-byte rows
    if (d->dtype == KGPU_F32 && K == 3 && off % 16)
      return set_error(KGPU_EINVAL, "f32 3-D leaf offset not a multiple of 16 bytes");
    if (len > 1024) return set_error(KGPU_EINVAL, "leaf longer than 1024 points");
    if (off + leaf_encoded_bytes(len, K, sa) > d->leaf_bytes_len)
      return set_error(KGPU_EINVAL, "leaf extent outside the arena");
    ex[2 * l] = uint32_t(off / 8);
    ex[2 * l + 1] = uint32_t(len);
    total += len;
  }
  if (total != d->size) return set_error(KGPU_EINVAL, "sum of leaf lengths != size");

  auto* t = new (std::nothrow) kgpu_tree();
  if (!t) return set_error(KGPU_ENOMEM, "host allocation failed");
  DeviceTree& dt = t->dt;
  dt.dtype = d->dtype;
  dt.dims = K;
  cudaGetDevice(&dt.device);
  dt.max_stem_level = d->max_stem_level;
  dt.leaf_count = uint32_t(d->leaf_count);
  dt.size = d->size;
  dt.stem_count = d->stem_count;
  dt.leaf_bytes_len = d->leaf_bytes_len;
  dt.max_leaf_len = d->max_leaf_len;
  dt.bh = donnelly ? d->block_height : 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // 3-D leaves are re-encoded as rows on the device.  f64 rows take 32 bytes
  // per point against 28 in the tiles, so they get offsets of their own (32 x
  // the points before the leaf) and the reference's extents stay beside them.
  const bool rows = K == 3 && d->leaf_bytes_len;
  const bool moved = rows && d->dtype == KGPU_F64;
  std::vector<uint32_t> rex;
  if (moved) {
    try {
      rex.resize(ex.size());
    } catch (const std::bad_alloc&) {
      delete t;
      return set_error(KGPU_ENOMEM, "host allocation failed");
    }
    uint64_t before = 0;
    for (uint64_t l = 0; l < d->leaf_count; ++l) {
      rex[2 * l] = uint32_t(before * 32 / 8);
      rex[2 * l + 1] = ex[2 * l + 1];
      before += ex[2 * l + 1];
    }
  }
  if (moved && d->size * 32 / 8 >= (uint64_t(1) << 32)) {
    delete t;
    return set_error(KGPU_EOVERFLOW, "f64 3-D rows larger than 32 GiB");
  }
  const size_t stem_bytes = std::max<size_t>(16, d->stem_count * sa);
  const size_t arena_bytes = std::max<size_t>(16, (moved ? d->size * 32 : d->leaf_bytes_len) + 16);
  const size_t ex_bytes = std::max<size_t>(16, ex.size() * 4);
  cudaError_t e;
  if ((e = cudaMalloc(&dt.stems, stem_bytes)) != cudaSuccess ||
      (e = cudaMalloc(reinterpret_cast<void**>(&dt.arena), arena_bytes)) != cudaSuccess ||
      (e = cudaMalloc(&dt.extents, ex_bytes)) != cudaSuccess ||
      (moved && (e = cudaMalloc(&dt.src_extents, ex_bytes)) != cudaSuccess)) {
    cudaFree(dt.stems);
    cudaFree(dt.arena);
    cudaFree(dt.extents);
    cudaFree(dt.src_extents);
    delete t;
    if (e == cudaErrorMemoryAllocation) return set_error(KGPU_ENOMEM, "device allocation failed");
    return cuda_fail(e, "cudaMalloc");
  }
  dt.device_bytes = stem_bytes + arena_bytes + ex_bytes * (moved ? 2 : 1);
  if (d->stem_count) e = cudaMemcpyAsync(dt.stems, d->stems, d->stem_count * sa, cudaMemcpyHostToDevice, s);
  // 3-D leaves are staged as tiles and re-encoded as rows on the device
  DevBuf tiles;
  if (e == cudaSuccess && rows) e = tiles.alloc(d->leaf_bytes_len, s);
  if (e == cudaSuccess && d->leaf_bytes_len)
    e = cudaMemcpyAsync(rows ? tiles.as<uint8_t>() : dt.arena, d->leaf_bytes, d->leaf_bytes_len,
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !ex.empty())
    e = cudaMemcpyAsync(dt.extents, moved ? rex.data() : ex.data(), ex.size() * 4,
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && moved)
    e = cudaMemcpyAsync(dt.src_extents, ex.data(), ex.size() * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && rows) e = convert_leaf_layout(dt, tiles.as<uint8_t>(), dt.arena, true, s);
  if (e == cudaSuccess && mapped) {
    dt.map_min = m->min_stem_leaf_idx;
    dt.map_len = uint32_t(lmap.size());
    if ((e = cudaMalloc(reinterpret_cast<void**>(&dt.leaf_map),
                        std::max<size_t>(16, lmap.size() * 4))) == cudaSuccess &&
        !lmap.empty())
      e = cudaMemcpyAsync(dt.leaf_map, lmap.data(), lmap.size() * 4, cudaMemcpyHostToDevice, s);
    dt.device_bytes += lmap.size() * 4;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // `ex` and `lmap` are locals
  if (e != cudaSuccess) {
    kgpu_tree_destroy(t);
    return cuda_fail(e, "uploading the tree");
  }
  *out = t;
  return KGPU_OK;
}

}  // namespace
}  // namespace kgpu

extern "C" {

int32_t kgpu_tree_create(const kgpu_tree_desc* d, void* stream, kgpu_tree** out) {
  return create_tree(d, nullptr, stream, out);
}

int32_t kgpu_tree_create_mapped(const kgpu_tree_desc* d, const kgpu_leaf_map* map, void* stream,
                                kgpu_tree** out) {
  if (!map) return set_error(KGPU_EINVAL, "NULL leaf map");
  return create_tree(d, map, stream, out);
}

}  // extern "C"

namespace kgpu {
namespace {
int create_flatvec(const kgpu_flatvec_desc* d, const kgpu_leaf_map* map, void* stream,
                   kgpu_tree** out) {
  if (!d || !out) return set_error(KGPU_EINVAL, "NULL argument");
  *out = nullptr;
  if (d->abi_version != KGPU_ABI_VERSION) return set_error(KGPU_EINVAL, "abi_version mismatch");
  Layout L;
  const int st = flatvec_to_layout(L, d->dtype, int(d->dims), d->columns, d->items, d->extents,
                                   d->leaf_count, d->size);
  if (st != KGPU_OK) return st;
  kgpu_tree_desc td;
  std::memset(&td, 0, sizeof(td));
  td.abi_version = KGPU_ABI_VERSION;
  td.dtype = d->dtype;
  td.dims = d->dims;
  td.item_size = 4;
  td.bucket_size = 32;
  td.stem_strategy = d->stem_strategy;
  td.block_height = d->block_height;
  td.resolution = map ? KGPU_RES_MAPPED : KGPU_RES_ARITHMETIC;
  td.stems = d->stems;
  td.stem_count = d->stem_count;
  td.leaf_bytes = L.leaf_bytes.data();
  td.leaf_bytes_len = L.leaf_bytes.size();
  td.leaf_extents = L.extents.data();
  td.leaf_count = d->leaf_count;
  td.max_stem_level = d->max_stem_level;
  td.size = d->size;
  td.max_leaf_len = L.max_leaf_len;
  return create_tree(&td, map, stream, out);
}

int create_vecofarrays(const kgpu_vecofarrays_desc* d, const kgpu_leaf_map* map, void* stream,
                       kgpu_tree** out) {
  if (!d || !out) return set_error(KGPU_EINVAL, "NULL argument");
  *out = nullptr;
  if (d->abi_version != KGPU_ABI_VERSION) return set_error(KGPU_EINVAL, "abi_version mismatch");
  if (d->dtype != KGPU_F32 && d->dtype != KGPU_F64) return set_error(KGPU_EINVAL, "unknown dtype");
  if (d->dims < 1 || d->dims > uint32_t(kMaxDims))
    return set_error(KGPU_EINVAL, "dims must be 1..4");
  if (d->bucket < 1 || d->bucket > 65536) return set_error(KGPU_EINVAL, "bucket must be 1..65536");
  if (d->leaf_count && (!d->content_points || !d->content_items || !d->sizes))
    return set_error(KGPU_EINVAL, "NULL leaf arrays");
  const uint64_t B = d->bucket;
  const uint32_t K = d->dims;
  uint64_t n = 0;
  for (uint64_t l = 0; l < d->leaf_count; ++l) {
    if (d->sizes[l] > B) return set_error(KGPU_EINVAL, "a leaf's size exceeds its bucket");
    n += d->sizes[l];
  }
  if (n >= 0xFFFFFFFFull) return set_error(KGPU_EOVERFLOW, "2^32 - 1 points or more");
  // gather the live slots into the FlatVec form: K columns, items, (start, end)
  const size_t esz = d->dtype == KGPU_F64 ? 8 : 4;
  std::vector<std::vector<uint8_t>> cols(K, std::vector<uint8_t>(n * esz));
  std::vector<uint32_t> items(n);
  std::vector<uint32_t> ext(2 * d->leaf_count);
  const uint8_t* pts = static_cast<const uint8_t*>(d->content_points);
  uint64_t at = 0;
  for (uint64_t l = 0; l < d->leaf_count; ++l) {
    const uint64_t len = d->sizes[l];
    for (uint32_t k = 0; k < K; ++k)
      std::memcpy(cols[k].data() + at * esz, pts + ((l * K + k) * B) * esz, len * esz);
    std::memcpy(items.data() + at, d->content_items + l * B, len * 4);
    ext[2 * l] = uint32_t(at);
    ext[2 * l + 1] = uint32_t(at + len);
    at += len;
  }
  kgpu_flatvec_desc f;
  std::memset(&f, 0, sizeof(f));
  f.abi_version = KGPU_ABI_VERSION;
  f.dtype = d->dtype;
  f.dims = K;
  f.stem_strategy = d->stem_strategy;
  f.block_height = d->block_height;
  f.max_stem_level = d->max_stem_level;
  f.stems = d->stems;
  f.stem_count = d->stem_count;
  for (uint32_t k = 0; k < K; ++k) f.columns[k] = cols[k].data();
  f.items = items.data();
  f.extents = ext.data();
  f.leaf_count = d->leaf_count;
  f.size = n;
  return create_flatvec(&f, map, stream, out);
}
}  // namespace
}  // namespace kgpu

extern "C" {

int32_t kgpu_tree_create_flatvec(const kgpu_flatvec_desc* d, void* stream, kgpu_tree** out) {
  return create_flatvec(d, nullptr, stream, out);
}

int32_t kgpu_tree_create_vecofarrays(const kgpu_vecofarrays_desc* d, void* stream,
                                     kgpu_tree** out) {
  return create_vecofarrays(d, nullptr, stream, out);
}

int32_t kgpu_tree_create_vecofarrays_mapped(const kgpu_vecofarrays_desc* d,
                                            const kgpu_leaf_map* map, void* stream,
                                            kgpu_tree** out) {
  if (!map) return set_error(KGPU_EINVAL, "NULL leaf map");
  return create_vecofarrays(d, map, stream, out);
}

int32_t kgpu_tree_destroy(kgpu_tree* t) {
  if (!t) return KGPU_OK;
  release_tree_arrays(t->dt);
  delete t;
  return KGPU_OK;
}

int32_t kgpu_tree_info(const kgpu_tree* t, int64_t* info) {
  if (!t || !info) return set_error(KGPU_EINVAL, "NULL argument");
  const DeviceTree& d = t->dt;
  info[0] = d.dtype;
  info[1] = d.dims;
  info[2] = int64_t(d.size);
  info[3] = int64_t(d.leaf_count);
  info[4] = d.max_stem_level;
  info[5] = int64_t(d.stem_count);
  info[6] = int64_t(d.leaf_bytes_len);
  info[7] = int64_t(d.device_bytes);
  return KGPU_OK;
}

}  // extern "C"

namespace kgpu {

int check_query_desc(const kgpu_tree* t, const kgpu_query_desc* d, bool radius_family) {
  if (!t || !d) return set_error(KGPU_EINVAL, "NULL argument");
  if (d->abi_version != KGPU_ABI_VERSION) return set_error(KGPU_EINVAL, "abi_version mismatch");
  if (d->metric < KGPU_SQUARED_EUCLIDEAN || d->metric > KGPU_MINKOWSKI4)
    return set_error(KGPU_EINVAL, "unknown metric");
  const int f = d->family;
  if (radius_family) {
    if (f != KGPU_WITHIN && f != KGPU_WITHIN_UNSORTED)
      return set_error(KGPU_EINVAL, "family is not a radius family");
  } else {
    if (f != KGPU_NEAREST_ONE && f != KGPU_APPROX_NEAREST_ONE && f != KGPU_NEAREST_N &&
        f != KGPU_NEAREST_N_WITHIN && f != KGPU_BEST_N_WITHIN)
      return set_error(KGPU_EINVAL, "family is not a fixed-size family");
    if (f == KGPU_NEAREST_N || f == KGPU_NEAREST_N_WITHIN || f == KGPU_BEST_N_WITHIN) {
      if (d->max_qty == 0) return set_error(KGPU_EINVAL, "max_qty must be >= 1");
      // The reference's collectors are unbounded (BinaryHeap above its
      // ThresholdVec range).  2-D and 3-D trees hold lists of any length up
      // to kMaxRowK in the output rows; the warp engine of 1-D and 4-D trees
      // keeps them in shared memory, up to kMaxBigK entries, Cartesian only.
      const bool rows = t->dt.dims == 2 || t->dt.dims == 3;
      if (d->max_qty > uint32_t(kMaxRowK))
        return set_error(KGPU_EUNSUPPORTED, "max_qty above 1,048,576 is not supported");
      if (!rows && d->max_qty > uint32_t(d->periodic_box ? kMaxK : kMaxBigK))
        return set_error(KGPU_EUNSUPPORTED,
                         d->periodic_box
                             ? "periodic max_qty above 32 is served for 2-D and 3-D trees"
                             : "max_qty above 256 is served for 2-D and 3-D trees");
    }
  }
  if (t->dt.scalar_walk()) {
    // Donnelly stems and Mapped resolution run the scalar backtracking walk
    // of the thread engine (2-D and 3-D trees).
    if (t->dt.dims != 2 && t->dt.dims != 3)
      return set_error(KGPU_EUNSUPPORTED,
                       "Donnelly and Mapped trees are served for 2-D and 3-D points");
    if (d->flags & KGPU_FLAG_ENGINE_WARP)
      return set_error(KGPU_EUNSUPPORTED, "Donnelly and Mapped trees run on the thread engine");
  }
  if (d->periodic_box) {
    // builder.rs: periodic queries support nearest_one, nearest_n(.within) and
    // within; best_n_within and approx are Cartesian-only.
    if (f == KGPU_BEST_N_WITHIN || f == KGPU_APPROX_NEAREST_ONE)
      return set_error(KGPU_EINVAL, "periodic boundaries apply to nearest_one, nearest_n and within");
    // PeriodicAxis::periodic_box_is_valid (builder.rs:29-35): every axis > 0
    for (int a = 0; a < t->dt.dims; ++a) {
      const double v = t->dt.dtype == KGPU_F64 ? static_cast<const double*>(d->periodic_box)[a]
                                               : double(static_cast<const float*>(d->periodic_box)[a]);
      if (!(v > 0.0)) return set_error(KGPU_EINVAL, "periodic box sizes must be strictly positive");
    }
  }
  return KGPU_OK;
}

// Whether nearest_n rows come out sorted by distance.  An unsorted request
// keeps arrival order only where the reference's collector is a ThresholdVec
// (max_qty <= MAX_UNSORTED_VEC_RESULT_SIZE = 24, nearest_n_within.rs:27); above
// that it collects into a BinaryHeap, whose into_vec order is unspecified, and
// the rows come out sorted (as the oracle restates it).
bool rows_sorted(const kgpu_query_desc* d) { return d->sorted != 0 || d->max_qty > 24; }

// Leaf-grouped processing order: forced on or off by the flags, otherwise on
// for batches large enough to share leaves (it never changes results).
bool want_spatial_order(uint32_t flags, uint64_t nq, uint64_t leaves) {
  if (nq < 2 || (flags & KGPU_FLAG_NO_SPATIAL_ORDER)) return false;
  if (flags & KGPU_FLAG_SPATIAL_ORDER) return true;
  return nq >= 65536 && leaves >= 4096;
}

void apply_periodic(const DeviceTree& dt, const kgpu_query_desc* d, QueryLaunch& q) {
  q.periodic = d->periodic_box != nullptr;
  if (!q.periodic) return;
  for (int a = 0; a < dt.dims; ++a)
    q.box[a] = dt.dtype == KGPU_F64 ? static_cast<const double*>(d->periodic_box)[a]
                                    : double(static_cast<const float*>(d->periodic_box)[a]);
}

// The lane-refilled kernels take their next chunk of queries from a device
// counter when they are given one: a warp whose chunks finish early takes
// more, where a fixed interleaved share of the batch left warps idle behind
// the slowest (kNN16 over 16M queries: 471M against 531M queries/s).  Forest
// batches bring their own counter; every other launch gets a fresh zeroed
// one, so launches never share a count.
template <typename F>
cudaError_t with_work_counter(const QueryLaunch& q, F&& launch) {
  if (q.work) return launch(q);
  DevBuf w;
  cudaError_t e = w.alloc(sizeof(unsigned long long), q.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(w.p, 0, sizeof(unsigned long long), q.stream);
  if (e != cudaSuccess) return e;
  QueryLaunch qw = q;
  qw.work = w.as<unsigned long long>();
  return launch(qw);
}

template <typename A>
cudaError_t launch_fixed(const DeviceTree& t, const QueryLaunch& q) {
  // thread engine for 2-D/3-D trees; periodic nearest_one stays on the warp
  // engine (home query plus images)
  // lists above 32 entries: nearest_n up to kMaxThreadK stays on the thread
  // engine (per-thread lists in 128-thread blocks: 136M against 62M queries/s
  // at k = 33 on C2's data, 42M against 36M at 64); larger k (the warp engine
  // was faster from k = 100), and best_n_within above 32, run on the warp
  // engine's shared-memory lists
  // Lists beyond those ranges live in the output rows (launch_trow): above
  // 256 entries, periodic nearest_n above 32, and Donnelly trees above 32.
  const bool nn = q.family == KGPU_NEAREST_N || q.family == KGPU_NEAREST_N_WITHIN;
  const bool best = q.family == KGPU_BEST_N_WITHIN;
  const bool two_three = t.dims == 2 || t.dims == 3;
  if ((nn || best) && two_three && q.k > kMaxK &&
      (q.k > kMaxBigK || (nn && q.periodic) || t.scalar_walk()))
    return with_work_counter(q, [&](const QueryLaunch& qw) { return launch_trow<A>(t, qw); });
  const bool big_k = q.k > kMaxK && (best || (nn && (q.k > kMaxThreadK || q.periodic)));
  const bool thread = (t.scalar_walk() || q.engine != 1) && two_three &&
                      (!q.periodic || q.family != KGPU_NEAREST_ONE || t.scalar_walk()) && !big_k;
  // the warp engine keeps its fixed shares: it takes one query at a time
  if (!thread) return launch_wfixed<A>(t, q);
  return with_work_counter(q, [&](const QueryLaunch& qw) { return launch_tfixed<A>(t, qw); });
}
template cudaError_t launch_fixed<float>(const DeviceTree&, const QueryLaunch&);
template cudaError_t launch_fixed<double>(const DeviceTree&, const QueryLaunch&);

namespace {


// With KGPU_FLAG_SPATIAL_ORDER, group the batch by straight-descent leaf and
// hand the kernels that processing order (same results, better locality).
cudaError_t maybe_spatial_order(const DeviceTree& dt, const kgpu_query_desc* d, QueryLaunch& q,
                                DevBuf& ob, DevBuf& sb, cudaStream_t s) {
  if (!want_spatial_order(d->flags, q.nq, q.forest ? q.total_leaves : dt.leaf_count))
    return cudaSuccess;
  cudaError_t e;
  if ((e = ob.alloc(q.nq * 4, s)) != cudaSuccess) return e;
  if ((e = sb.alloc(spatial_order_scratch_bytes(dt, q), s)) != cudaSuccess) return e;
  e = dt.dtype == KGPU_F64 ? launch_spatial_order<double>(dt, q, ob.as<uint32_t>(), sb.p)
                           : launch_spatial_order<float>(dt, q, ob.as<uint32_t>(), sb.p);
  if (e == cudaSuccess) q.order = ob.as<uint32_t>();
  return e;
}

template <typename A>
cudaError_t run_fixed(const DeviceTree& dt, QueryLaunch& q) {
  bool handled = false;
  const cudaError_t e = periodic_fast<A>(dt, q, handled);
  return handled ? e : launch_fixed<A>(dt, q);
}

int out_width(const kgpu_query_desc* d) {
  return (d->family == KGPU_NEAREST_ONE || d->family == KGPU_APPROX_NEAREST_ONE)
             ? 1
             : int(d->max_qty);
}

// Counts the rows of a nearest_n chunk holding fewer than `full` entries
// (min(k, size); a row falls short only when its query's distances are NaN,
// which no candidate passes, or the tree's points hold NaN).
__global__ void k_short_rows(const uint32_t* __restrict__ counts, uint64_t n, uint32_t full,
                             uint32_t* __restrict__ out) {
  uint32_t m = 0;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x)
    m += counts[i] != full ? 1u : 0u;
  m = __reduce_add_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(out, m);
}

#ifndef KGPU_HOST_SLOTS
#define KGPU_HOST_SLOTS 3
#endif
#ifndef KGPU_HOST_CHUNK_LOG2
#define KGPU_HOST_CHUNK_LOG2 21
#endif
#ifndef KGPU_HOST_EDGE_DIV
#define KGPU_HOST_EDGE_DIV 8
#endif
// Host buffers: the batch goes through in 2M-query chunks on three internal
// streams, each with its own device buffers, so the copy of one chunk's
// queries in, another chunk's kernel and a third chunk's results out run at
// the same time (full overlap needs pinned host memory).  With two slots a
// chunk's kernel waited for the results of the chunk two back to leave its
// buffers; on kNN16 over 16M queries, three slots took the call from 55.8 to
// 49.1 ms, against 36.9 ms for the result copy alone.  Work already queued on
// the caller's stream runs first; the call returns when every result is on
// the host.
int query_host_pipelined(const DeviceTree& dt, const kgpu_query_desc* d, const QueryLaunch& base,
                         const void* queries, uint64_t nq, int w, void* out_dists,
                         uint32_t* out_items, uint32_t* out_counts, cudaStream_t s) {
  const size_t sa = dt.dtype == KGPU_F64 ? 8 : 4;
  constexpr int kSlots = KGPU_HOST_SLOTS;
  const uint64_t chunk = std::min<uint64_t>(nq, uint64_t(1) << KGPU_HOST_CHUNK_LOG2);
  const int nslots = int(std::min<uint64_t>(kSlots, (nq + chunk - 1) / chunk));
  cudaStream_t st[kSlots] = {};
  // nearest_n without a radius fills min(k, size) entries in every row whose
  // query has comparable distances, so those counts are written on the host
  // while the device works instead of crossing the bus.  The rows' counts stay
  // on the device (all_counts), a small kernel counts each chunk's rows short
  // of that, and only chunks with such rows are copied back at the end.
  uint32_t* const host_counts = out_counts;
  const bool counts_known = out_counts && d->family == KGPU_NEAREST_N;
  const uint32_t full = uint32_t(std::min<uint64_t>(uint64_t(w), dt.size));
  const uint64_t edge = std::max<uint64_t>(1, chunk / KGPU_HOST_EDGE_DIV);
  const uint64_t max_chunks = (nq + edge - 1) / edge + 1;
  DevBuf all_counts, short_rows;
  std::vector<std::pair<uint64_t, uint64_t>> spans;  // (first query, length) per chunk
  cudaError_t e = cudaSuccess;
  if (counts_known) {
    out_counts = nullptr;
    if ((e = all_counts.alloc(nq * 4, s)) == cudaSuccess &&
        (e = short_rows.alloc(max_chunks * 4, s)) == cudaSuccess)
      e = cudaMemsetAsync(short_rows.p, 0, max_chunks * 4, s);
  }
  auto count_short_rows = [&](uint64_t c0, uint64_t nc, uint64_t ci, cudaStream_t ss) {
    k_short_rows<<<148 * 2, 256, 0, ss>>>(all_counts.as<uint32_t>() + c0, nc, full,
                                          short_rows.as<uint32_t>() + ci);
    ++g_launches;
    return cudaGetLastError();
  };
  cudaEvent_t ready = nullptr;
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(ready, s);
  for (int i = 0; i < nslots && e == cudaSuccess; ++i) {
    e = cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st[i], ready, 0);
  }
  int status = KGPU_OK;
  if (e != cudaSuccess) status = cuda_fail(e, "creating the copy streams");
  {
    DevBuf bq[kSlots], bd[kSlots], bi[kSlots], bc[kSlots], bord[kSlots], bos[kSlots];
    for (int i = 0; i < nslots && status == KGPU_OK; ++i) {
      if ((e = bq[i].alloc(chunk * dt.dims * sa, st[i])) != cudaSuccess ||
          (e = bd[i].alloc(chunk * w * sa, st[i])) != cudaSuccess ||
          (e = bi[i].alloc(chunk * w * 4, st[i])) != cudaSuccess ||
          (out_counts && (e = bc[i].alloc(chunk * 4, st[i])) != cudaSuccess))
        status = e == cudaErrorMemoryAllocation ? set_error(KGPU_ENOMEM, "device allocation failed")
                                                : cuda_fail(e, "cudaMallocAsync");
    }
    // The first and the last chunk are short (an eighth of a chunk): the first
    // chunk's kernel runs before any result can leave, and the last chunk's
    // results leave after every kernel, so shorter ends shorten the
    // unoverlapped head and tail (kNN16 over 16M queries: 50.9 -> 47.1 ms).
    auto chunk_len = [&](uint64_t c0) -> uint64_t {
      const uint64_t rem = nq - c0;
      if (nslots == 1 || rem <= edge) return rem;
      if (c0 == 0) return edge;
      if (rem <= chunk + edge) return rem - edge;
      return chunk;
    };
    uint64_t nc = 0;
    for (uint64_t c0 = 0, ci = 0; c0 < nq && status == KGPU_OK; c0 += nc, ++ci) {
      const int slot = int(ci % nslots);
      cudaStream_t ss = st[slot];
      nc = chunk_len(c0);
      QueryLaunch q = base;
      q.nq = nc;
      q.queries = bq[slot].p;
      q.out_d = bd[slot].p;
      q.out_i = bi[slot].as<uint32_t>();
      q.out_c = counts_known ? all_counts.as<uint32_t>() + c0
                             : out_counts ? bc[slot].as<uint32_t>() : nullptr;
      q.stream = ss;
      const char* what = nullptr;
      if ((e = cudaMemcpyAsync(bq[slot].p, static_cast<const uint8_t*>(queries) + c0 * dt.dims * sa,
                               nc * dt.dims * sa, cudaMemcpyHostToDevice, ss)) != cudaSuccess) {
        what = "copying queries to the device";
      } else {
        // the order buffers of the previous chunk on this slot are freed on
        // this stream, after that chunk's kernel
        bord[slot].~DevBuf();
        new (&bord[slot]) DevBuf();
        bos[slot].~DevBuf();
        new (&bos[slot]) DevBuf();
        if ((e = maybe_spatial_order(dt, d, q, bord[slot], bos[slot], ss)) != cudaSuccess)
          what = "ordering the batch";
        else if ((e = dt.dtype == KGPU_F64 ? run_fixed<double>(dt, q) : run_fixed<float>(dt, q)) !=
                 cudaSuccess)
          what = "launching the query kernel";
        else if (counts_known && (e = count_short_rows(c0, nc, ci, ss)) != cudaSuccess)
          what = "checking the rows' counts";
        else if ((e = cudaMemcpyAsync(static_cast<uint8_t*>(out_dists) + c0 * w * sa, bd[slot].p,
                                      nc * w * sa, cudaMemcpyDeviceToHost, ss)) != cudaSuccess ||
                 (e = cudaMemcpyAsync(out_items + c0 * w, bi[slot].p, nc * w * 4,
                                      cudaMemcpyDeviceToHost, ss)) != cudaSuccess ||
                 (out_counts && (e = cudaMemcpyAsync(out_counts + c0, bc[slot].p, nc * 4,
                                                     cudaMemcpyDeviceToHost, ss)) != cudaSuccess))
          what = "copying results to the host";
      }
      if (what) status = cuda_fail(e, what);
      spans.emplace_back(c0, nc);
    }
    if (counts_known && status == KGPU_OK) std::fill(host_counts, host_counts + nq, full);
    for (int i = 0; i < nslots; ++i)
      if (st[i] && (e = cudaStreamSynchronize(st[i])) != cudaSuccess && status == KGPU_OK)
        status = cuda_fail(e, "query execution");
    if (counts_known && status == KGPU_OK) {
      // the chunks with short rows, if any, bring their counts back
      std::vector<uint32_t> shorts(spans.size());
      e = cudaMemcpy(shorts.data(), short_rows.p, spans.size() * 4, cudaMemcpyDeviceToHost);
      for (size_t i = 0; i < spans.size() && e == cudaSuccess; ++i)
        if (shorts[i])
          e = cudaMemcpy(host_counts + spans[i].first, all_counts.as<uint32_t>() + spans[i].first,
                         spans[i].second * 4, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) status = cuda_fail(e, "copying results to the host");
    }
  }  // device buffers are released on their streams here
  for (int i = 0; i < nslots; ++i)
    if (st[i]) {
      cudaStreamSynchronize(st[i]);
      cudaStreamDestroy(st[i]);
    }
  if (ready) cudaEventDestroy(ready);
  return status;
}

}  // namespace
}  // namespace kgpu

extern "C" {

int32_t kgpu_query(kgpu_tree* t, const kgpu_query_desc* d, const void* queries, uint64_t nq,
                   void* out_dists, uint32_t* out_items, uint32_t* out_counts, void* stream) {
  int st = check_query_desc(t, d, false);
  if (st != KGPU_OK) return st;
  if (nq == 0) return KGPU_OK;
  if (!queries || !out_dists || !out_items) return set_error(KGPU_EINVAL, "NULL buffer");
  const DeviceTree& dt = t->dt;
  const int w = out_width(d);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  QueryLaunch q;
  q.family = d->family;
  q.metric = d->metric;
  q.k = w;
  q.radius = (d->family == KGPU_NEAREST_N) ? __builtin_inf() : d->radius;
  q.exclusive = d->exclusive != 0;
  q.sorted = rows_sorted(d);
  q.nq = nq;
  apply_periodic(dt, d, q);
  q.engine = engine_of(d->flags);
  apply_tuning(d->tuning, q);
  const bool host = (d->flags & KGPU_FLAG_HOST_BUFFERS) != 0;
  cudaError_t e = cudaSuccess;
  if (host) return query_host_pipelined(dt, d, q, queries, nq, w, out_dists, out_items, out_counts, s);
  q.queries = queries;
  q.out_d = out_dists;
  q.out_i = out_items;
  q.out_c = out_counts;
  q.stream = s;
  DevBuf bord, bos;
  if ((e = maybe_spatial_order(dt, d, q, bord, bos, s)) != cudaSuccess)
    return cuda_fail(e, "ordering the batch");
  e = dt.dtype == KGPU_F64 ? run_fixed<double>(dt, q) : run_fixed<float>(dt, q);
  if (e != cudaSuccess) return cuda_fail(e, "launching the query kernel");
  return KGPU_OK;
}

int32_t kgpu_query_radius_count(kgpu_tree* t, const kgpu_query_desc* d, const void* queries,
                                uint64_t nq, uint64_t* offsets, void* stream) {
  int st = check_query_desc(t, d, true);
  if (st != KGPU_OK) return st;
  if (!offsets) return set_error(KGPU_EINVAL, "offsets is NULL");
  if (nq > 0 && !queries) return set_error(KGPU_EINVAL, "queries is NULL");
  const DeviceTree& dt = t->dt;
  const size_t sa = dt.dtype == KGPU_F64 ? 8 : 4;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool host = (d->flags & KGPU_FLAG_HOST_BUFFERS) != 0;
  DevBuf bq, boff, btmp;
  cudaError_t e;
  QueryLaunch q;
  q.family = d->family;
  q.metric = d->metric;
  q.radius = d->radius;
  q.exclusive = d->exclusive != 0;
  q.sorted = d->family == KGPU_WITHIN && d->sorted != 0;
  q.nq = nq;
  apply_periodic(dt, d, q);
  q.engine = engine_of(d->flags);
  apply_tuning(d->tuning, q);
  q.stream = s;
  uint64_t* doff = offsets;
  if (host) {
    if ((e = bq.alloc(nq * dt.dims * sa, s)) != cudaSuccess ||
        (e = boff.alloc((nq + 1) * 8, s)) != cudaSuccess)
      return set_error(KGPU_ENOMEM, "device allocation failed");
    if (nq && (e = cudaMemcpyAsync(bq.p, queries, nq * dt.dims * sa, cudaMemcpyHostToDevice, s)) !=
                  cudaSuccess)
      return cuda_fail(e, "copying queries to the device");
    q.queries = bq.p;
    doff = boff.as<uint64_t>();
  } else {
    q.queries = queries;
  }
  if ((e = btmp.alloc(scan_tmp_bytes(nq), s)) != cudaSuccess)
    return set_error(KGPU_ENOMEM, "device allocation failed");
  DevBuf bord, bos;
  if ((e = maybe_spatial_order(dt, d, q, bord, bos, s)) != cudaSuccess)
    return cuda_fail(e, "ordering the batch");
  if (nq) {
    e = dt.dtype == KGPU_F64 ? launch_within_count<double>(dt, q, doff)
                             : launch_within_count<float>(dt, q, doff);
    if (e != cudaSuccess) return cuda_fail(e, "launching the counting kernel");
  }
  e = launch_exclusive_scan(doff, doff, nq, btmp.p, s);
  if (e != cudaSuccess) return cuda_fail(e, "launching the scan");
  if (host) {
    if ((e = cudaMemcpyAsync(offsets, doff, (nq + 1) * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return cuda_fail(e, "copying offsets to the host");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "radius count");
  }
  return KGPU_OK;
}

int32_t kgpu_query_radius_fill(kgpu_tree* t, const kgpu_query_desc* d, const void* queries,
                               uint64_t nq, const uint64_t* offsets, void* out_dists,
                               uint32_t* out_items, void* stream) {
  int st = check_query_desc(t, d, true);
  if (st != KGPU_OK) return st;
  if (!offsets) return set_error(KGPU_EINVAL, "offsets is NULL");
  if (nq == 0) return KGPU_OK;
  if (!queries) return set_error(KGPU_EINVAL, "queries is NULL");
  const DeviceTree& dt = t->dt;
  const size_t sa = dt.dtype == KGPU_F64 ? 8 : 4;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool host = (d->flags & KGPU_FLAG_HOST_BUFFERS) != 0;
  const bool sorted = d->family == KGPU_WITHIN && d->sorted != 0;
  uint64_t total = 0;
  cudaError_t e;
  if (host) {
    total = offsets[nq];
  } else {
    if ((e = cudaMemcpyAsync(&total, offsets + nq, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return cuda_fail(e, "reading the hit total");
  }
  if (total == 0) return KGPU_OK;
  if (!out_dists || !out_items) return set_error(KGPU_EINVAL, "NULL output buffer");
  DevBuf bq, boff, bd, bi, sd, si;
  QueryLaunch q;
  q.family = d->family;
  q.metric = d->metric;
  q.radius = d->radius;
  q.exclusive = d->exclusive != 0;
  q.sorted = sorted;
  q.nq = nq;
  apply_periodic(dt, d, q);
  q.engine = engine_of(d->flags);
  apply_tuning(d->tuning, q);
  q.stream = s;
  const uint64_t* doff = offsets;
  if (host) {
    if ((e = bq.alloc(nq * dt.dims * sa, s)) != cudaSuccess ||
        (e = boff.alloc((nq + 1) * 8, s)) != cudaSuccess ||
        (e = bd.alloc(total * sa, s)) != cudaSuccess || (e = bi.alloc(total * 4, s)) != cudaSuccess)
      return set_error(KGPU_ENOMEM, "device allocation failed");
    if ((e = cudaMemcpyAsync(bq.p, queries, nq * dt.dims * sa, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(boff.p, offsets, (nq + 1) * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return cuda_fail(e, "copying inputs to the device");
    q.queries = bq.p;
    doff = boff.as<uint64_t>();
    q.out_d = bd.p;
    q.out_i = bi.as<uint32_t>();
  } else {
    q.queries = queries;
    q.out_d = out_dists;
    q.out_i = out_items;
  }
  DevBuf bord, bos;
  if ((e = maybe_spatial_order(dt, d, q, bord, bos, s)) != cudaSuccess)
    return cuda_fail(e, "ordering the batch");
  e = dt.dtype == KGPU_F64 ? launch_within_fill<double>(dt, q, doff)
                           : launch_within_fill<float>(dt, q, doff);
  if (e != cudaSuccess) return cuda_fail(e, "launching the fill kernel");
  if (sorted) {
    if ((e = sd.alloc(total * sa, s)) != cudaSuccess || (e = si.alloc(total * 4, s)) != cudaSuccess)
      return set_error(KGPU_ENOMEM, "device allocation failed");
    e = dt.dtype == KGPU_F64
            ? launch_seg_sort<double>(doff, nq, total, static_cast<double*>(q.out_d), q.out_i,
                                      sd.as<double>(), si.as<uint32_t>(), s)
            : launch_seg_sort<float>(doff, nq, total, static_cast<float*>(q.out_d), q.out_i,
                                     sd.as<float>(), si.as<uint32_t>(), s);
    if (e != cudaSuccess) return cuda_fail(e, "launching the segmented sort");
  }
  if (host) {
    if ((e = cudaMemcpyAsync(out_dists, q.out_d, total * sa, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(out_items, q.out_i, total * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return cuda_fail(e, "copying results to the host");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "radius fill");
  }
  return KGPU_OK;
}

int32_t kgpu_query_stats(kgpu_tree* t, const kgpu_query_desc* d, const void* queries, uint64_t nq,
                         uint64_t* stats, void* stream) {
  if (!t || !d || !stats) return set_error(KGPU_EINVAL, "NULL argument");
  const bool radius = d->family == KGPU_WITHIN || d->family == KGPU_WITHIN_UNSORTED;
  int st = check_query_desc(t, d, radius);
  if (st != KGPU_OK) return st;
  stats[0] = stats[1] = stats[2] = 0;
  if (nq == 0) return KGPU_OK;
  if (!queries) return set_error(KGPU_EINVAL, "queries is NULL");
  const DeviceTree& dt = t->dt;
  const size_t sa = dt.dtype == KGPU_F64 ? 8 : 4;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool host = (d->flags & KGPU_FLAG_HOST_BUFFERS) != 0;
  const int w = radius ? 1 : out_width(d);
  DevBuf bq, bd, bi, bst;
  cudaError_t e;
  if ((e = bd.alloc(radius ? (nq + 1) * 8 : nq * w * sa, s)) != cudaSuccess ||
      (e = bi.alloc(nq * w * 4, s)) != cudaSuccess || (e = bst.alloc(3 * 8, s)) != cudaSuccess)
    return set_error(KGPU_ENOMEM, "device allocation failed");
  const void* dq = queries;
  if (host) {
    if ((e = bq.alloc(nq * dt.dims * sa, s)) != cudaSuccess)
      return set_error(KGPU_ENOMEM, "device allocation failed");
    if ((e = cudaMemcpyAsync(bq.p, queries, nq * dt.dims * sa, cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
      return cuda_fail(e, "copying queries to the device");
    dq = bq.p;
  }
  if ((e = cudaMemsetAsync(bst.p, 0, 24, s)) != cudaSuccess) return cuda_fail(e, "memset");
  QueryLaunch q;
  q.family = d->family;
  q.metric = d->metric;
  q.k = w;
  q.radius = (d->family == KGPU_NEAREST_N) ? __builtin_inf() : d->radius;
  q.exclusive = d->exclusive != 0;
  q.sorted = d->sorted != 0;
  q.nq = nq;
  apply_periodic(dt, d, q);
  q.engine = engine_of(d->flags);
  apply_tuning(d->tuning, q);
  q.queries = dq;
  q.out_d = bd.p;
  q.out_i = bi.as<uint32_t>();
  q.stats = bst.as<unsigned long long>();
  q.stream = s;
  if (radius)
    e = dt.dtype == KGPU_F64 ? launch_within_count<double>(dt, q, bd.as<uint64_t>())
                             : launch_within_count<float>(dt, q, bd.as<uint64_t>());
  else
    e = dt.dtype == KGPU_F64 ? run_fixed<double>(dt, q) : run_fixed<float>(dt, q);
  if (e != cudaSuccess) return cuda_fail(e, "launching the query kernel");
  if ((e = cudaMemcpyAsync(stats, bst.p, 24, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return cuda_fail(e, "reading statistics");
  return KGPU_OK;
}

}  // extern "C"
