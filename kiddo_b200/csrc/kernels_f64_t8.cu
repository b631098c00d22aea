// kernels_f64_t8.cu — thread-per-query kernels with a 8-slot list for double coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_THREAD(double, 8)
