// kernels_f64.cu — query-engine kernels instantiated for double coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE(double)
