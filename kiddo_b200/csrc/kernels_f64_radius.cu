// kernels_f64_radius.cu — radius and ordering kernels instantiated for double coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_RADIUS(double)
