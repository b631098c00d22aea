// kernels_f32_t1.cu — thread-per-query kernels with a 1-slot list for float coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_THREAD(float, 1)
