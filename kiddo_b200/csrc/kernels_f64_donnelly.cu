// kernels_f64_donnelly.cu — thread-per-query kernels over Donnelly stems (scalar
// backtracking), double coordinates: fixed-size families and the radius passes.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_DONNELLY(double)
