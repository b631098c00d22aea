// kernels_f32_warp.cu — warp-per-query fixed-size kernels (periodic included) for float coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_WARP(float)
