// kernels_f32_thread.cu — thread-per-query fixed-size kernels for float coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_THREAD(float)
