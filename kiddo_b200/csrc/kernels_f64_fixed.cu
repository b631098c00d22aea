// kernels_f64_fixed.cu — fixed-size kernels instantiated for double coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_FIXED(double)
