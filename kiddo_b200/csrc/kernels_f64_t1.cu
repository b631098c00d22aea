// kernels_f64_t1.cu — thread-per-query kernels with a 1-slot list for double coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_THREAD(double, 1)
