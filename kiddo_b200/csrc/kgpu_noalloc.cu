// kgpu_noalloc.cu — the counting pass of a radius query without any allocation.
//
// Why: some callers of this library cannot allocate device memory while they
// query.  A serving process that reserves all of HBM for its own pool at start
// up has nothing left for cudaMalloc/cudaMallocAsync; a latency-critical loop
// must not pay for (or synchronise on) an allocation; a host framework whose
// allocator owns every device buffer forbids allocations behind its back.
// kgpu_query_radius_count needs a little scratch for its prefix sum (one
// 64-bit total per tile of 2048 queries), which it takes from the
// stream-ordered allocator.  This entry point takes the same scratch from a
// fixed array in device memory that the library carries instead.
//
// The array lives in this file as a file-scope __device__ variable.  Every GPU
// on which the library is loaded holds it (64 KiB) until the process exits.
// In host code its name is only a host-side stand-in, not a device address, so
// the host code below asks the runtime for the device address once per device
// (cudaGetSymbolAddress, with that device current) and passes that address to
// the scan kernels.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/kiddo_gpu.h"
#include "kgpu_internal.h"
#include "kgpu_launch.h"
#include "kgpu_tree_impl.h"

namespace kgpu {
namespace {

// Largest batch the fixed scratch can serve: 2^24 queries (the scan keeps one
// u64 per 2048 queries plus the grand total).
constexpr uint64_t kNoAllocMaxQueries = uint64_t(1) << 24;
constexpr uint64_t kNoAllocScratchWords = kNoAllocMaxQueries / 2048 + 1;

static __device__ __align__(256) unsigned long long g_noalloc_scan_tiles[kNoAllocScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct CachedAddress {
  uint64_t ctx_id = 0;  // the context the address was looked up in
  void* addr = nullptr;
};
CachedAddress g_scratch_addr[kMaxDevices];

// Device address of g_noalloc_scan_tiles on the current device.  It is looked
// up once per device and context: cudaDeviceReset destroys the context that
// holds the array, and the next call looks the address up again in the new
// one.  Returns nullptr and sets the error message on failure.
void* scratch_address(int dev) {
  const uint64_t ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_mu);
  CachedAddress& c = g_scratch_addr[dev];
  if (!c.addr || c.ctx_id != ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scan_tiles);
    if (e != cudaSuccess || !p) {
      set_error(KGPU_ECUDA, std::string("cudaGetSymbolAddress of the scan scratch: ") +
                                cudaGetErrorString(e));
      return nullptr;
    }
    c.addr = p;
    c.ctx_id = ctx;
  }
  return c.addr;
}

}  // namespace
}  // namespace kgpu

using namespace kgpu;

extern "C" int32_t kgpu_query_radius_count_noalloc(kgpu_tree* t, const kgpu_query_desc* d,
                                                   const void* queries, uint64_t nq,
                                                   uint64_t* offsets, void* stream) {
  int st = check_query_desc(t, d, true);
  if (st != KGPU_OK) return st;
  if (d->flags & KGPU_FLAG_HOST_BUFFERS)
    return set_error(KGPU_EINVAL,
                     "the no-allocation count takes device pointers only (host buffers "
                     "would need staging allocations)");
  if (!offsets) return set_error(KGPU_EINVAL, "offsets is NULL");
  if (nq > 0 && !queries) return set_error(KGPU_EINVAL, "queries is NULL");
  if (nq > kNoAllocMaxQueries || scan_tmp_bytes(nq) > sizeof(g_noalloc_scan_tiles))
    return set_error(KGPU_EOVERFLOW,
                     "batch larger than the no-allocation limit of 16,777,216 queries; split "
                     "it or use kgpu_query_radius_count");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(KGPU_ECUDA, cudaGetErrorString(e));
  if (dev != t->dt.device)
    return set_error(KGPU_EINVAL, "the tree's device must be the current device");
  if (dev < 0 || dev >= kMaxDevices) return set_error(KGPU_EUNSUPPORTED, "device index too large");
  void* tiles = scratch_address(dev);
  if (!tiles) return KGPU_ECUDA;

  const DeviceTree& dt = t->dt;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
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
  q.queries = queries;
  q.stream = s;
  if (nq) {
    e = dt.dtype == KGPU_F64 ? launch_within_count<double>(dt, q, offsets)
                             : launch_within_count<float>(dt, q, offsets);
    if (e != cudaSuccess) return set_error(KGPU_ECUDA, cudaGetErrorString(e));
  }
  // Every tile total the scan reads is written earlier in the same call, so
  // nothing in the shared scratch has to start at zero.
  e = launch_exclusive_scan(offsets, offsets, nq, tiles, s);
  if (e != cudaSuccess) return set_error(KGPU_ECUDA, cudaGetErrorString(e));
  return KGPU_OK;
}
