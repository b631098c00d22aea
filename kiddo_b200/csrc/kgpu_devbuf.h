// kgpu_devbuf.h — stream-ordered scratch buffers of the library's entry points.
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

namespace kgpu {

// Stream-ordered allocation from the library's own memory pool on the current
// device (one per device and context, created on first use).  The pool keeps
// freed scratch cached across stream synchronizations (release threshold at
// its maximum), so a call does not map memory that the previous call just
// gave back; the device's default pool is left as it was.  kgpu_scratch_trim
// returns the cached memory to the driver.
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s);

// The pool scratch_alloc draws from on `dev` (made if needed).
cudaError_t library_pool(int dev, cudaMemPool_t* out);

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
