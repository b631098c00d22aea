// kgpu_periodic_fast.cu — periodic nearest_n through a plain walk where the
// box's faces cannot change the answer.
//
// The reference answers a periodic nearest_n with one walk under min-image
// distances (kd_tree/query/periodic.rs:455-619).  For a query whose final
// list (or radius) keeps clear of every face of the box, that answer is the
// plain walk's answer, bit for bit:
//  * a point's min-image distance differs from its plain distance only when
//    wrapping shortens some axis a, and the wrapped offset on that axis is then
//    at least face_a = min(q_a, box_a - q_a) when every point lies in
//    [0, box) (c_a > q_a: box_a - (c_a - q_a) > q_a; c_a < q_a:
//    box_a - q_a + c_a >= box_a - q_a); each axis term adds a non-negative
//    amount, so such a point's periodic distance is at least the metric's
//    axis term of face_a;
//  * when that term is above the plain list's bound (its k-th distance, or
//    the radius while the list is not full), no wrapped point reaches the
//    list, and every point that does has the same distance, computed by the
//    same operations, either way (the min-image offset of an unwrapped axis is
//    |q_a - c_a| itself);
//  * both walks visit leaves depth first, near child first, so the points
//    both visit arrive in the same relative order, and equal distances keep
//    the same one.  The sorted list is the k smallest by (distance, arrival)
//    either way.
// So the batch runs the plain walk first, a small kernel lists the queries
// whose bound comes within a safety margin of a face (or whose coordinates
// are not inside the box), and the periodic walk runs on those alone,
// overwriting their rows.  Batches that ask for the warp engine keep its
// periodic walk for every row.  Unsorted lists are not taken this way (their order
// after evictions depends on every insertion the walk made), nor are
// traversal statistics (they count the reference's periodic walk).
#include <algorithm>
#include <cstdint>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "kgpu_device.cuh"
#include "kgpu_devbuf.h"
#include "kgpu_launch.h"
#include "kgpu_launch_impl.cuh"

namespace kgpu {
namespace {

// Per-block minimum and maximum of every axis over the stored points (out:
// gridDim.x rows of 2K values), and a flag for any NaN coordinate.
template <typename A, int K>
__global__ void __launch_bounds__(256) k_point_bounds(TreeView<A> tv, A* __restrict__ out,
                                                      int* __restrict__ nan_seen) {
  A lo[K], hi[K];
#pragma unroll
  for (int d = 0; d < K; ++d) {
    lo[d] = inf_of<A>();
    hi[d] = -inf_of<A>();
  }
  bool nan = false;
  for (uint64_t l = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; l < tv.leaf_count;
       l += uint64_t(gridDim.x) * blockDim.x) {
    const uint2 ex = __ldg(tv.extents + l);
    const uint8_t* base = tv.arena + size_t(ex.x) * 8;
    for (uint32_t p = 0; p < ex.y; ++p) {
      A c[K];
      uint32_t item;
      load_point<A, K>(base, ex.y, p, c, item);
#pragma unroll
      for (int d = 0; d < K; ++d) {
        nan |= c[d] != c[d];
        lo[d] = c[d] < lo[d] ? c[d] : lo[d];
        hi[d] = c[d] > hi[d] ? c[d] : hi[d];
      }
    }
  }
  __shared__ A red[2 * K][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < K; ++d) {
    for (int o = 16; o > 0; o >>= 1) {
      const A a = __shfl_xor_sync(0xffffffffu, lo[d], o);
      const A b = __shfl_xor_sync(0xffffffffu, hi[d], o);
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = b > hi[d] ? b : hi[d];
    }
    if (lane == 0) {
      red[d][warp] = lo[d];
      red[K + d][warp] = hi[d];
    }
  }
  if (__any_sync(0xffffffffu, nan) && lane == 0) atomicOr(nan_seen, 1);
  __syncthreads();
  if (threadIdx.x < 2 * K) {
    const int j = threadIdx.x;
    A v = red[j][0];
    for (int w = 1; w < int(blockDim.x >> 5); ++w) {
      const A x = red[j][w];
      v = j < K ? (x < v ? x : v) : (x > v ? x : v);
    }
    out[size_t(blockIdx.x) * 2 * K + j] = v;
  }
}

// Lists the queries the plain walk's answer cannot stand for: some axis's
// face term, less a margin for rounding, is not above the row's bound, or a
// coordinate is not strictly inside the box (NaN included).  The margins: an
// absolute 8 units in the last place of the box size on the face (the
// computed wrapped offset can fall short of the exact one by a few), then a
// relative 1e-5 on the axis term.
template <typename A, int K, typename M>
__global__ void __launch_bounds__(256) k_periodic_needed(
    const A* __restrict__ Q, uint64_t nq, const A* __restrict__ out_d,
    const uint32_t* __restrict__ out_c, int k, A radius, BoxArg<A, K> box,
    uint32_t* __restrict__ list, unsigned long long* __restrict__ count) {
  constexpr A kUlps = sizeof(A) == 4 ? A(8.0 / 8388608.0) : A(8.0 / 4503599627370496.0);
  constexpr A kShrink = A(1.0 - 1e-5);
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < nq;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const A bound = out_c[i] >= uint32_t(k) ? out_d[i * uint64_t(k) + uint64_t(k - 1)] : radius;
    bool clear = true;
#pragma unroll
    for (int d = 0; d < K; ++d) {
      const A q = Q[i * K + d];
      const A up = sub_rn(box.v[d], q);
      const A face = sub_rn(q < up ? q : up, mul_rn(box.v[d], kUlps));
      clear = clear && face > A(0) && mul_rn(M::template dist1<A>(face, A(0)), kShrink) > bound;
    }
    if (!clear) list[atomicAdd(count, 1ull)] = uint32_t(i);
  }
}

std::mutex g_bounds_mu;

// The stored points' per-axis bounds, measured once per tree on a stream of
// its own (false when they cannot be measured now: the caller's stream is
// being captured into a graph, or a CUDA call failed).
template <typename A>
bool point_bounds(const DeviceTree& dt, cudaStream_t caller) {
  std::lock_guard<std::mutex> g(g_bounds_mu);
  if (dt.point_bounds >= 0) return dt.point_bounds == 1;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(caller, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return false;
  if (dt.size == 0 || dt.leaf_count == 0) {
    dt.point_bounds = 0;
    return false;
  }
  const int K = dt.dims;
  const int blocks = 148 * 2;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return false;
  // after the work already on the caller's stream (a pending upload included)
  cudaEvent_t ev = nullptr;
  bool ok = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventRecord(ev, caller) == cudaSuccess && cudaStreamWaitEvent(s, ev, 0) == cudaSuccess;
  void* buf = nullptr;
  ok = ok && cudaMalloc(&buf, size_t(blocks) * 2 * K * sizeof(A) + 16) == cudaSuccess;
  int* nan_seen = reinterpret_cast<int*>(static_cast<uint8_t*>(buf) +
                                         size_t(blocks) * 2 * K * sizeof(A));
  ok = ok && cudaMemsetAsync(nan_seen, 0, sizeof(int), s) == cudaSuccess;
  if (ok) {
    const TreeView<A> tv = make_view<A>(dt);
    ok = with_dims(K, [&](auto kk) -> cudaError_t {
           constexpr int KK = decltype(kk)::value;
           k_point_bounds<A, KK><<<blocks, 256, 0, s>>>(tv, static_cast<A*>(buf), nan_seen);
           ++g_launches;
           return cudaGetLastError();
         }) == cudaSuccess;
  }
  std::vector<A> rows(size_t(blocks) * 2 * K);
  int nan = 0;
  ok = ok &&
       cudaMemcpyAsync(rows.data(), buf, rows.size() * sizeof(A), cudaMemcpyDeviceToHost, s) ==
           cudaSuccess &&
       cudaMemcpyAsync(&nan, nan_seen, sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
       cudaStreamSynchronize(s) == cudaSuccess;
  if (buf) cudaFree(buf);
  if (ev) cudaEventDestroy(ev);
  cudaStreamDestroy(s);
  if (!ok) return false;
  for (int d = 0; d < K; ++d) {
    double lo = double(rows[d]), hi = double(rows[K + d]);
    for (int b = 1; b < blocks; ++b) {
      lo = std::min(lo, double(rows[size_t(b) * 2 * K + d]));
      hi = std::max(hi, double(rows[size_t(b) * 2 * K + K + d]));
    }
    dt.point_lo[d] = lo;
    dt.point_hi[d] = hi;
  }
  dt.point_bounds = nan ? 0 : 1;
  return dt.point_bounds == 1;
}

}  // namespace

// Batches below this size go straight to the periodic walk: the plain pass,
// the check and the second launch cost more than they save there.
constexpr uint64_t kFastMinBatch = uint64_t(1) << 16;

template <typename A>
cudaError_t periodic_fast(const DeviceTree& dt, const QueryLaunch& q, bool& handled) {
  handled = false;
  const bool nn = q.family == KGPU_NEAREST_N || q.family == KGPU_NEAREST_N_WITHIN;
  if (!q.periodic || !nn || !q.sorted || q.stats || q.forest || q.radii || q.nq_dev ||
      q.engine == 1 || dt.scalar_walk() || (dt.dims != 2 && dt.dims != 3) ||
      q.nq < kFastMinBatch)
    return cudaSuccess;
  if (!point_bounds<A>(dt, q.stream)) return cudaSuccess;
  for (int d = 0; d < dt.dims; ++d) {
    const double box = double(A(q.box[d]));
    if (!(dt.point_lo[d] >= 0.0) || !(dt.point_hi[d] < box)) return cudaSuccess;
  }
  handled = true;
  cudaError_t e;
  // 1. the plain walk for every query (counts into scratch if the caller
  //    asked for none)
  DevBuf counts, list, n_listed;
  QueryLaunch qp = q;
  qp.periodic = false;
  if (!qp.out_c) {
    if ((e = counts.alloc(q.nq * 4, q.stream)) != cudaSuccess) return e;
    qp.out_c = counts.as<uint32_t>();
  }
  if ((e = launch_fixed<A>(dt, qp)) != cudaSuccess) return e;
  // 2. the queries whose rows the box's faces could change
  if ((e = list.alloc(q.nq * 4, q.stream)) != cudaSuccess ||
      (e = n_listed.alloc(8, q.stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(n_listed.p, 0, 8, q.stream)) != cudaSuccess)
    return e;
  e = with_dims(dt.dims, [&](auto kk) -> cudaError_t {
    constexpr int K = decltype(kk)::value;
    return with_metric(q.metric, [&](auto m) -> cudaError_t {
      using M = decltype(m);
      const uint64_t blocks = std::min<uint64_t>((q.nq + 255) / 256, 148 * 8);
      k_periodic_needed<A, K, M><<<unsigned(blocks), 256, 0, q.stream>>>(
          static_cast<const A*>(q.queries), q.nq, static_cast<const A*>(q.out_d), qp.out_c, q.k,
          A(q.radius), make_box<A, K>(q), list.as<uint32_t>(),
          n_listed.as<unsigned long long>());
      ++g_launches;
      return cudaGetLastError();
    });
  });
  if (e != cudaSuccess) return e;
  // 3. the periodic walk over the listed queries alone, overwriting their rows
  QueryLaunch qq = q;
  qq.order = list.as<uint32_t>();
  qq.nq_dev = n_listed.as<unsigned long long>();
  return launch_fixed<A>(dt, qq);
}
template cudaError_t periodic_fast<float>(const DeviceTree&, const QueryLaunch&, bool&);
template cudaError_t periodic_fast<double>(const DeviceTree&, const QueryLaunch&, bool&);

}  // namespace kgpu
