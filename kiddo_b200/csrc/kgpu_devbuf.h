// kgpu_devbuf.h — stream-ordered scratch buffers of the library's entry points.
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

namespace kgpu {

// cudaMallocAsync from the current device's default memory pool.  On a
// device's first use the pool's release threshold is raised to its maximum,
// so that freed scratch stays cached in the pool across stream
// synchronizations instead of going back to the driver at each one (and being
// mapped again, milliseconds later, by the next call).  This is a setting of
// the process's default pool: other cudaMallocAsync users in the process see
// the same caching.
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s);

struct DeviceTree;
// Frees a tree's stems, arena, extents and point table, from the pool (DeviceTree::pooled)
// or from cudaMalloc, after the device's pending work.
void release_tree_arrays(DeviceTree& dt);

// RAII scratch buffer, released on its stream.
struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  cudaError_t alloc(size_t bytes, cudaStream_t st) {
    s = st;
    return scratch_alloc(&p, bytes ? bytes : 16, st);
  }
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFreeAsync(p, s);
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace kgpu
