// Step kernel instantiations for D2Q9 (one translation unit per lattice keeps
// the build parallel).
#include "step_kernels.cuh"

LBM_INSTANTIATE_STEP(D2Q9, LBM_F32)
LBM_INSTANTIATE_STEP(D2Q9, LBM_F64)
LBM_INSTANTIATE_STEP(D2Q9, LBM_F16)
LBM_INSTANTIATE_STEP(D2Q9, LBM_BF16)
