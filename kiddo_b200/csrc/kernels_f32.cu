// kernels_f32.cu — query-engine kernels instantiated for float coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE(float)
