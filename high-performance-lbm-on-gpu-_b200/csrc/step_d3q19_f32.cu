// Step kernel instantiations for D3Q19, f32 storage.
#include "step_kernels.cuh"

LBM_INSTANTIATE_STEP(D3Q19, LBM_F32)
