// kernels_f32_t8.cu — thread-per-query kernels with a 8-slot list for float coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_THREAD(float, 8)
