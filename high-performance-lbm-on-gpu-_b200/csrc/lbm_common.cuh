// Shared device code of the B200 LBM kernels: lattice tables, storage formats,
// node kinds and the TRT + Guo collision.
//
// Lattice direction order and weights are those of the reference solver
// (src/lbm/lattice.py:114-146), so population slot k means the same direction
// on both sides of the C ABI.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lbm_b200.h"

namespace lbm {

// ---------------------------------------------------------------- node kinds
// One byte per node. SOLID nodes are never updated. SPECIAL fluid nodes carry
// link rules, an immersed-boundary force or rule-term exports and are updated
// by the boundary warps from a compact list; the bulk threads skip them.
// NEAR marks fluid nodes with at least one solid neighbour: only they test
// their neighbours' kinds. EDGE marks fluid nodes on a face of the box, whose
// neighbours wrap periodically. A node with kind 0 is interior: it streams
// with fixed, warp-uniform offsets and no branch at all.
constexpr uint8_t KIND_FLUID = 0;
constexpr uint8_t KIND_SOLID = LBM_KIND_SOLID;
constexpr uint8_t KIND_SPECIAL = LBM_KIND_SPECIAL;
constexpr uint8_t KIND_NEAR = LBM_KIND_NEAR;
constexpr uint8_t KIND_EDGE = LBM_KIND_EDGE;

// ---------------------------------------------------------------- lattices
// Tables are constexpr functions of a direction index: every direction loop
// is fully unrolled, the index folds to a constant and f[Q] stays in registers.
struct D2Q9 {
    static constexpr int D = 2;
    static constexpr int Q = 9;
    __host__ __device__ static constexpr int cx(int i) { return (i == 1 || i == 5 || i == 8) ? 1 : (i == 3 || i == 6 || i == 7) ? -1 : 0; }
    __host__ __device__ static constexpr int cy(int i) { return (i == 2 || i == 5 || i == 6) ? 1 : (i == 4 || i == 7 || i == 8) ? -1 : 0; }
    __host__ __device__ static constexpr int cz(int) { return 0; }
    __host__ __device__ static constexpr int opp(int i) { return i == 0 ? 0 : (i <= 4 ? ((i + 1) & 3) + 1 : ((i - 3) & 3) + 5); }
    __host__ __device__ static constexpr double w(int i) { return i == 0 ? 4.0 / 9.0 : (i <= 4 ? 1.0 / 9.0 : 1.0 / 36.0); }
};

struct D3Q19 {
    static constexpr int D = 3;
    static constexpr int Q = 19;
    // Axis links 1..6 as (+x,-x,+y,-y,+z,-z); edge links 7..18 in pairs
    // (xy: 7..10, xz: 11..14, yz: 15..18), each next to its opposite.
    __host__ __device__ static constexpr int cx(int i) {
        return (i == 1 || i == 7 || i == 9 || i == 11 || i == 13) ? 1 : (i == 2 || i == 8 || i == 10 || i == 12 || i == 14) ? -1 : 0;
    }
    __host__ __device__ static constexpr int cy(int i) {
        return (i == 3 || i == 7 || i == 10 || i == 15 || i == 17) ? 1 : (i == 4 || i == 8 || i == 9 || i == 16 || i == 18) ? -1 : 0;
    }
    __host__ __device__ static constexpr int cz(int i) {
        return (i == 5 || i == 11 || i == 14 || i == 15 || i == 18) ? 1 : (i == 6 || i == 12 || i == 13 || i == 16 || i == 17) ? -1 : 0;
    }
    __host__ __device__ static constexpr int opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
    __host__ __device__ static constexpr double w(int i) { return i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18.0 : 1.0 / 36.0); }
};

// ---------------------------------------------------------------- storage
// Populations are stored shifted (f~ = f - w). Float16 storage multiplies by
// a power of two before rounding so that small f~ stay out of the subnormal
// range; the scale is exact in both directions.
constexpr float FP16_SCALE = 16384.0f;  // 2^14
constexpr float FP16_INV_SCALE = 1.0f / 16384.0f;

template <int ST> struct Storage;

template <> struct Storage<LBM_F32> {
    using T = float;
    using R = float;
    __device__ static __forceinline__ R load(const T* p) { return *p; }
    __device__ static __forceinline__ R load_nc(const T* p) { return __ldg(p); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = v; }
    __device__ static __forceinline__ R round(R v) { return v; }
    __device__ static __forceinline__ T encode(R v) { return v; }
    __device__ static __forceinline__ R decode(T v) { return v; }
};

template <> struct Storage<LBM_F64> {
    using T = double;
    using R = double;
    __device__ static __forceinline__ R load(const T* p) { return *p; }
    __device__ static __forceinline__ R load_nc(const T* p) { return __ldg(p); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = v; }
    __device__ static __forceinline__ R round(R v) { return v; }
    __device__ static __forceinline__ T encode(R v) { return v; }
    __device__ static __forceinline__ R decode(T v) { return v; }
};

template <> struct Storage<LBM_F16> {
    using T = __half;
    using R = float;
    __device__ static __forceinline__ R decode(T v) { return __half2float(v) * FP16_INV_SCALE; }
    __device__ static __forceinline__ T encode(R v) { return __float2half_rn(v * FP16_SCALE); }
    __device__ static __forceinline__ R load(const T* p) { return decode(*p); }
    __device__ static __forceinline__ R load_nc(const T* p) { return decode(__ldg(p)); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = encode(v); }
    __device__ static __forceinline__ R round(R v) { return decode(encode(v)); }
};

template <> struct Storage<LBM_BF16> {
    using T = __nv_bfloat16;
    using R = float;
    __device__ static __forceinline__ R decode(T v) { return __bfloat162float(v); }
    __device__ static __forceinline__ T encode(R v) { return __float2bfloat16_rn(v); }
    __device__ static __forceinline__ R load(const T* p) { return decode(*p); }
    __device__ static __forceinline__ R load_nc(const T* p) { return decode(__ldg(p)); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = encode(v); }
    __device__ static __forceinline__ R round(R v) { return decode(encode(v)); }
};

// ---------------------------------------------------------------- collision
// TRT + Guo forcing on one node (reference src/lbm/collision.py:59-88,
// forcing.py:37-56). With rho = 1 + sum f~, u = (sum c f + F/2)/rho and, for
// each opposite pair (i, o = opp i), cu = c_i.u and cF = c_i.F, the update
//   f*_i = f_i - w+ (f+ - feq+) - w- (f- - feq-) + S+ + S-
// (f+- = (f_i +- f_o)/2, feq+ = w (drho + rho (4.5 cu^2 - 1.5 u.u)),
//  feq- = 3 w rho cu, S+ = w (1 - w+/2)(9 cu cF - 3 u.F), S- = 3 w (1 - w-/2) cF)
// is evaluated in factored form
//   f*_i = a f_i + b f_o + E + O,   f*_o = a f_o + b f_i + E - O
//   a = 1 - (w+ + w-)/2,  b = (w- - w+)/2
//   E = w (A + cu (B cu + C cF)),  O = w (D cu + G cF)
//   A = w+ (drho - 1.5 rho u.u) - 3 (1 - w+/2) u.F,  B = 4.5 w+ rho,  C = 9 (1 - w+/2)
//   D = 3 w- rho,  G = 3 (1 - w-/2)
// so each pair costs ~15 operations; the node-level scalars are shared. BGK
// is w- = w+ (b = 0). The rest population: f*_0 = (1 - w+) f_0 + w_0 A.
template <class L, class R>
__device__ __forceinline__ void collide(R (&f)[L::Q], R wp, R wm, R Fx, R Fy, R Fz)
{
    R drho = f[0], jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        drho += f[i];
        if (L::cx(i) > 0) jx += f[i];
        if (L::cx(i) < 0) jx -= f[i];
        if (L::cy(i) > 0) jy += f[i];
        if (L::cy(i) < 0) jy -= f[i];
        if (L::cz(i) > 0) jz += f[i];
        if (L::cz(i) < 0) jz -= f[i];
    }
    const R rho = R(1) + drho;
    const R inv = R(1) / rho;
    const R ux = (jx + R(0.5) * Fx) * inv;
    const R uy = (jy + R(0.5) * Fy) * inv;
    const R uz = L::D == 3 ? (jz + R(0.5) * Fz) * inv : R(0);
    const R usq = ux * ux + uy * uy + uz * uz;
    const R uF = ux * Fx + uy * Fy + (L::D == 3 ? uz * Fz : R(0));
    const R ap = R(1) - R(0.5) * wp;
    const R am = R(1) - R(0.5) * wm;
    const R A = wp * (drho - R(1.5) * rho * usq) - R(3) * ap * uF;
    const R B = R(4.5) * wp * rho;
    const R C = R(9) * ap;
    const R Dm = R(3) * wm * rho;
    const R G = R(3) * am;
    const R ca = R(1) - R(0.5) * (wp + wm);
    const R cb = R(0.5) * (wm - wp);
    f[0] = (R(1) - wp) * f[0] + R(L::w(0)) * A;
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        const int o = L::opp(i);
        if (o < i) continue;
        const R wi = R(L::w(i));
        const R cu = R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz;
        const R cF = R(L::cx(i)) * Fx + R(L::cy(i)) * Fy + R(L::cz(i)) * Fz;
        const R E = wi * (A + cu * (B * cu + C * cF));
        const R O = wi * (Dm * cu + G * cF);
        const R fi = f[i], fo = f[o];
        f[i] = ca * fi + (cb * fo + (E + O));
        f[o] = ca * fo + (cb * fi + (E - O));
    }
}

// Moving-wall (Ladd) term 6 w_i (c_i . u_w) with u_w read at solid node s.
template <class L, class R>
__device__ __forceinline__ R wall_term(int i, const R* __restrict__ wall_u, int64_t s, int64_t qstride)
{
    if (wall_u == nullptr) return R(0);
    R cu = R(0);
    if (L::cx(i) != 0) cu += R(L::cx(i)) * wall_u[s];
    if (L::cy(i) != 0) cu += R(L::cy(i)) * wall_u[qstride + s];
    if (L::D == 3 && L::cz(i) != 0) cu += R(L::cz(i)) * wall_u[2 * qstride + s];
    return R(6) * R(L::w(i)) * cu;
}

__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// ---------------------------------------------------------------- arguments
// Everything one step launch needs, passed by value. Pointers to compute-type
// arrays are void* here and cast by the templated kernels.
struct StepArgs {
    int nx, ny, nz, pitch;
    int64_t qstride;  // elements between direction planes (pitch * ny * nz)
    double wp, wm, fx, fy, fz;
    const uint8_t* kind;
    const void* f_src;
    void* f_dst;
    const void* wall_u;
    const void* force_field;
    lbm_special_t sp;
    int32_t* status;
};

}  // namespace lbm
