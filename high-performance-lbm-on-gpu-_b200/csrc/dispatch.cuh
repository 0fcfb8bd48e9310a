// Run-time (lattice, storage) -> template dispatch for the C entry points.
#pragma once

#include "lbm_common.cuh"

namespace lbm {

template <class L, int ST> int launch_step(const StepArgs& a, int variant, int mode, int tile_x, int tile_y, cudaStream_t stream);
template <class L, int ST> int step_resources(int variant, int32_t* out4);

// Argument checks and StepArgs of the step entry points (abi.cu); launch may be null (defaults).
bool grid_valid(const lbm_grid_t* g);
bool special_valid(const lbm_special_t* sp, bool aa);
int make_args(StepArgs& a, const lbm_grid_t* g, const lbm_physics_t* p, const lbm_special_t* sp,
              const lbm_launch_t* launch, const uint8_t* kind, const void* src, void* dst, int& tx, int& ty, int& mode);

// Invoke FN<L, ST>(args...) for the run-time lattice and storage codes.
#define LBM_DISPATCH(lattice, storage, FN, ...)                                            \
    do {                                                                                   \
        const int _lat = (lattice), _st = (storage);                                       \
        if (_lat == LBM_D2Q9) {                                                            \
            switch (_st) {                                                                 \
            case LBM_F32: return FN<::lbm::D2Q9, LBM_F32>(__VA_ARGS__);                    \
            case LBM_F64: return FN<::lbm::D2Q9, LBM_F64>(__VA_ARGS__);                    \
            case LBM_F16: return FN<::lbm::D2Q9, LBM_F16>(__VA_ARGS__);                    \
            case LBM_BF16: return FN<::lbm::D2Q9, LBM_BF16>(__VA_ARGS__);                  \
            default: return LBM_ERR_INVALID;                                               \
            }                                                                              \
        } else if (_lat == LBM_D3Q19) {                                                    \
            switch (_st) {                                                                 \
            case LBM_F32: return FN<::lbm::D3Q19, LBM_F32>(__VA_ARGS__);                   \
            case LBM_F64: return FN<::lbm::D3Q19, LBM_F64>(__VA_ARGS__);                   \
            case LBM_F16: return FN<::lbm::D3Q19, LBM_F16>(__VA_ARGS__);                   \
            case LBM_BF16: return FN<::lbm::D3Q19, LBM_BF16>(__VA_ARGS__);                 \
            default: return LBM_ERR_INVALID;                                               \
            }                                                                              \
        }                                                                                  \
        return LBM_ERR_INVALID;                                                            \
    } while (0)

inline int launch_status() { return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH; }

inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace lbm
