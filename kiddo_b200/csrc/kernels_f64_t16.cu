// kernels_f64_t16.cu — thread-per-query kernels with a 16-slot list for double coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_THREAD(double, 16)
