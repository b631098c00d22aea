// kernels_f64_thread.cu — thread-per-query fixed-size kernels for double coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_THREAD(double)
