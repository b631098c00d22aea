// kernels_f32_radius.cu — radius and ordering kernels instantiated for float coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_RADIUS(float)
