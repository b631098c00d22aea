// kernels_f32_rows.cu — lists of any length in the output rows (float coordinates):
// nearest_n and best_n_within beyond the shared-memory kernels, Donnelly trees
// above 32 entries, periodic nearest_n.
#include "kgpu_launch_impl.cuh"

KGPU_INSTANTIATE_ROWS(float)
