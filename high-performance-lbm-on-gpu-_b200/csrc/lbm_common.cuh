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

// ---------------------------------------------------------------- stochastic rounding
// The step kernels store post-collision populations in 16-bit formats with
// stochastic rounding: a value between two neighbouring 16-bit numbers goes
// to the upper one with probability equal to its distance from the lower one
// (in units of their gap). Rounding then adds no bias, and a per-step change
// smaller than half a gap still accumulates; round-to-nearest drops such
// changes every step, which stalls slow or weakly forced flows.
// The random bits are a pure function of (node, step, direction), so runs are
// reproducible and the oracle replays them bit for bit:
//   h   = lowbias32(node ^ lowbias32(step)),   node = x + nx (y + ny z)
//   r_i = (h * sr_mult(i)) >> (32 - dropped bits)
// lowbias32 is the 32-bit integer hash published by C. Wellons
// (hash-prospector); the odd multipliers decorrelate the directions.
__host__ __device__ constexpr uint32_t sr_mult(int i) { return 0x9E3779B9u * (uint32_t)(2 * i + 1); }

__host__ __device__ __forceinline__ uint32_t lowbias32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ uint32_t sr_node_hash(int64_t natural, uint32_t step)
{
    return lowbias32((uint32_t)natural ^ lowbias32(step));
}

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
    static constexpr bool STOCHASTIC = false;
    __device__ static __forceinline__ R load(const T* p) { return *p; }
    __device__ static __forceinline__ R load_nc(const T* p) { return __ldg(p); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = v; }
    __device__ static __forceinline__ void store_sr(T* p, R v, uint32_t, int) { *p = v; }
    __device__ static __forceinline__ R round(R v) { return v; }
    __device__ static __forceinline__ R round_sr(R v, uint32_t, int) { return v; }
    __device__ static __forceinline__ T encode(R v) { return v; }
    __device__ static __forceinline__ R decode(T v) { return v; }
};

template <> struct Storage<LBM_F64> {
    using T = double;
    using R = double;
    static constexpr bool STOCHASTIC = false;
    __device__ static __forceinline__ R load(const T* p) { return *p; }
    __device__ static __forceinline__ R load_nc(const T* p) { return __ldg(p); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = v; }
    __device__ static __forceinline__ void store_sr(T* p, R v, uint32_t, int) { *p = v; }
    __device__ static __forceinline__ R round(R v) { return v; }
    __device__ static __forceinline__ R round_sr(R v, uint32_t, int) { return v; }
    __device__ static __forceinline__ T encode(R v) { return v; }
    __device__ static __forceinline__ R decode(T v) { return v; }
};

template <> struct Storage<LBM_F16> {
    using T = __half;
    using R = float;
    __device__ static __forceinline__ R decode(T v) { return __half2float(v) * FP16_INV_SCALE; }
    __device__ static __forceinline__ T encode(R v) { return __float2half_rn(v * FP16_SCALE); }
    // stochastic: add 13 random bits below the 10 kept mantissa bits of the
    // scaled float32, then truncate (exact in the normal float16 range)
    __device__ static __forceinline__ T encode_sr(R v, uint32_t h, int i)
    {
        const uint32_t b = __float_as_uint(v * FP16_SCALE) + ((h * sr_mult(i)) >> 19);
        return __float2half_rn(__uint_as_float(b & 0xFFFFE000u));
    }
    static constexpr bool STOCHASTIC = true;
    __device__ static __forceinline__ R load(const T* p) { return decode(*p); }
    __device__ static __forceinline__ R load_nc(const T* p) { return decode(__ldg(p)); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = encode(v); }
    __device__ static __forceinline__ void store_sr(T* p, R v, uint32_t h, int i) { *p = encode_sr(v, h, i); }
    __device__ static __forceinline__ R round(R v) { return decode(encode(v)); }
    __device__ static __forceinline__ R round_sr(R v, uint32_t h, int i) { return decode(encode_sr(v, h, i)); }
};

template <> struct Storage<LBM_BF16> {
    using T = __nv_bfloat16;
    using R = float;
    __device__ static __forceinline__ R decode(T v) { return __bfloat162float(v); }
    __device__ static __forceinline__ T encode(R v) { return __float2bfloat16_rn(v); }
    // stochastic: add 16 random bits below the kept half, then truncate
    __device__ static __forceinline__ T encode_sr(R v, uint32_t h, int i)
    {
        const uint32_t b = __float_as_uint(v) + ((h * sr_mult(i)) >> 16);
        return __ushort_as_bfloat16((unsigned short)(b >> 16));
    }
    static constexpr bool STOCHASTIC = true;
    __device__ static __forceinline__ R load(const T* p) { return decode(*p); }
    __device__ static __forceinline__ R load_nc(const T* p) { return decode(__ldg(p)); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = encode(v); }
    __device__ static __forceinline__ void store_sr(T* p, R v, uint32_t h, int i) { *p = encode_sr(v, h, i); }
    __device__ static __forceinline__ R round(R v) { return decode(encode(v)); }
    __device__ static __forceinline__ R round_sr(R v, uint32_t h, int i) { return decode(encode_sr(v, h, i)); }
};

// ---------------------------------------------------------------- arithmetic
// The collision is written once over a value type V (float or double).
// Every operation is an explicit round-to-nearest intrinsic, so the compiler
// never contracts or reorders it differently in different kernels: the bulk,
// boundary, fused and batched kernels give a node the same bits.
__device__ __forceinline__ float v_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float v_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float v_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float v_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float v_rcp(float a) { return __frcp_rn(a); }
__device__ __forceinline__ double v_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double v_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double v_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double v_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double v_rcp(double a) { return __drcp_rn(a); }

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
// u = (j + F/2) / rho uses one reciprocal per node.
template <class L, class V>
__device__ __forceinline__ void collide(V (&f)[L::Q], V wp, V wm,
                                        V Fx, V Fy, V Fz)
{
    const V zero = V(0);
    V drho = f[0], jx = zero, jy = zero, jz = zero;
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        drho = v_add(drho, f[i]);
        if (L::cx(i) > 0) jx = v_add(jx, f[i]);
        if (L::cx(i) < 0) jx = v_sub(jx, f[i]);
        if (L::cy(i) > 0) jy = v_add(jy, f[i]);
        if (L::cy(i) < 0) jy = v_sub(jy, f[i]);
        if (L::cz(i) > 0) jz = v_add(jz, f[i]);
        if (L::cz(i) < 0) jz = v_sub(jz, f[i]);
    }
    const V half = V(0.5);
    const V rho = v_add(V(1), drho);
    const V inv = v_rcp(rho);
    const V ux = v_mul(v_fma(half, Fx, jx), inv);
    const V uy = v_mul(v_fma(half, Fy, jy), inv);
    const V uz = L::D == 3 ? v_mul(v_fma(half, Fz, jz), inv) : zero;
    V usq = v_mul(ux, ux);
    usq = v_fma(uy, uy, usq);
    if (L::D == 3) usq = v_fma(uz, uz, usq);
    V uF = v_mul(ux, Fx);
    uF = v_fma(uy, Fy, uF);
    if (L::D == 3) uF = v_fma(uz, Fz, uF);
    // Node-independent constants, also with explicit rounding: a contracted
    // 1 - w/2 in one kernel and an uncontracted one in another would differ.
    const V ap = v_sub(V(1), v_mul(V(0.5), wp)), am = v_sub(V(1), v_mul(V(0.5), wm));
    // A = w+ (drho - 1.5 rho usq) - 3 ap uF
    const V A = v_fma(v_mul(V(-3), ap), uF, v_mul(wp, v_fma(v_mul(V(-1.5), rho), usq, drho)));
    const V B = v_mul(v_mul(V(4.5), wp), rho);
    const V C = v_mul(V(9), ap);
    const V Dm = v_mul(v_mul(V(3), wm), rho);
    const V G = v_mul(V(3), am);
    const V ca = v_sub(V(1), v_mul(V(0.5), v_add(wp, wm)));
    const V cb = v_mul(V(0.5), v_sub(wm, wp));
    f[0] = v_fma(v_sub(V(1), wp), f[0], v_mul(V(L::w(0)), A));
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        const int o = L::opp(i);
        if (o < i) continue;
        const V wi = V(L::w(i));
        // cu, cF: sums of +-components (exact sign flips, no multiplies)
        V cu = zero, cF = zero;
        bool first = true;
        if (L::cx(i) != 0) { cu = L::cx(i) > 0 ? ux : v_sub(zero, ux); cF = L::cx(i) > 0 ? Fx : v_sub(zero, Fx); first = false; }
        if (L::cy(i) != 0) {
            if (first) { cu = L::cy(i) > 0 ? uy : v_sub(zero, uy); cF = L::cy(i) > 0 ? Fy : v_sub(zero, Fy); first = false; }
            else { cu = L::cy(i) > 0 ? v_add(cu, uy) : v_sub(cu, uy); cF = L::cy(i) > 0 ? v_add(cF, Fy) : v_sub(cF, Fy); }
        }
        if (L::cz(i) != 0) {
            if (first) { cu = L::cz(i) > 0 ? uz : v_sub(zero, uz); cF = L::cz(i) > 0 ? Fz : v_sub(zero, Fz); }
            else { cu = L::cz(i) > 0 ? v_add(cu, uz) : v_sub(cu, uz); cF = L::cz(i) > 0 ? v_add(cF, Fz) : v_sub(cF, Fz); }
        }
        const V E = v_mul(wi, v_fma(cu, v_fma(B, cu, v_mul(C, cF)), A));
        const V O = v_mul(wi, v_fma(Dm, cu, v_mul(G, cF)));
        const V fi = f[i], fo = f[o];
        f[i] = v_fma(ca, fi, v_fma(cb, fo, v_add(E, O)));
        f[o] = v_fma(ca, fo, v_fma(cb, fi, v_sub(E, O)));
    }
}

// Moving-wall (Ladd) term 6 w_i (c_i . u_w) with u_w read at solid node s,
// in explicitly rounded operations (added with v_add by every caller), so
// every kernel that applies it gives the same bits.
template <class L, class R>
__device__ __forceinline__ R wall_term(int i, const R* __restrict__ wall_u, int64_t s, int64_t qstride)
{
    if (wall_u == nullptr) return R(0);
    R cu = R(0);
    if (L::cx(i) != 0) cu = v_add(cu, v_mul(R(L::cx(i)), wall_u[s]));
    if (L::cy(i) != 0) cu = v_add(cu, v_mul(R(L::cy(i)), wall_u[qstride + s]));
    if (L::D == 3 && L::cz(i) != 0) cu = v_add(cu, v_mul(R(L::cz(i)), wall_u[2 * qstride + s]));
    return v_mul(R(6.0 * L::w(i)), cu);
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
    const uint32_t* nbr;  // solid-neighbour mask per node
    // Step counter of the stochastic rounding (16-bit storage): the launch
    // reads seed[parity] and its bulk part writes seed[parity ^ 1] = +1.
    uint32_t* seed;
    int parity;
    lbm_special_t sp;
};

// The bulk (or fused) launch of a step advances the step counter: one thread
// writes the other slot, which no thread of this step reads.
__device__ __forceinline__ void advance_seed(const StepArgs& a)
{
    if (a.seed != nullptr && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 &&
        threadIdx.y == 0)
        a.seed[a.parity ^ 1] = a.seed[a.parity] + 1u;
}

}  // namespace lbm
