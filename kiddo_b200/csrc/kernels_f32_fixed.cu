// kernels_f32_fixed.cu — fixed-size kernels instantiated for float coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_FIXED(float)
