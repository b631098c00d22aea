// kernels_f64_warp.cu — warp-per-query fixed-size kernels (periodic included) for double coordinates.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_WARP(double)
