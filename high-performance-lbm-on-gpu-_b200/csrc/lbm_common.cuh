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
// The rounding is Blackwell's cvt.rs: a float32 v goes to the 16-bit format
// by adding R units of 2^-13 (float16; 2^-16 for bfloat16) of the
// destination spacing at |v| to |v| and truncating toward zero; float16
// magnitudes that reach 65536 become infinite. One instruction converts two
// values, taking R from bits 0-12 (0-15) of a 32-bit random word for the
// lower half and bits 16-28 (16-31) for the upper half. Nodes pair up along x
// (x even with x + 1) and share one word per direction:
//   pair = (z ny + y) ceil(nx / 2) + floor(x / 2),  h = lowbias32(pair ^ lowbias32(step))
//   word_i = (h ^ K_i) * 0x9E3779B9,  K_i = lowbias32(i + 1)
// the even node taking the lower half's bits, the odd node the upper half's.
// It is a pure function of (node, step, direction): runs are reproducible and
// the oracle replays them bit for bit. lowbias32 is the 32-bit integer hash
// published by C. Wellons (hash-prospector).
__host__ __device__ constexpr uint32_t lowbias32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__host__ __device__ constexpr uint32_t sr_key(int i) { return lowbias32((uint32_t)i + 1u); }
constexpr uint32_t SR_MULT = 0x9E3779B9u;

__device__ __forceinline__ int64_t sr_pair(int nx, int ny, int x, int y, int z)
{
    return ((int64_t)z * ny + y) * ((nx + 1) >> 1) + (x >> 1);
}
__device__ __forceinline__ uint32_t sr_pair_hash(int64_t pair, uint32_t step)
{
    return lowbias32((uint32_t)pair ^ lowbias32(step));
}
__device__ __forceinline__ uint32_t sr_word(uint32_t h, int i) { return (h ^ sr_key(i)) * SR_MULT; }

// d = (16-bit hi : 16-bit lo), stochastically rounded with rbits
__device__ __forceinline__ uint32_t cvt_rs_f16x2(float hi, float lo, uint32_t rbits)
{
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}
__device__ __forceinline__ uint32_t cvt_rs_bf16x2(float hi, float lo, uint32_t rbits)
{
    uint32_t d;
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
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
    static constexpr int SCALE_LOG2 = 0;
    __device__ static __forceinline__ R load(const T* p) { return *p; }
    __device__ static __forceinline__ R load_nc(const T* p) { return __ldg(p); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = v; }
    __device__ static __forceinline__ void store_sr(T* p, R v, uint32_t, int, bool) { *p = v; }
    __device__ static __forceinline__ R round(R v) { return v; }
    __device__ static __forceinline__ R round_sr(R v, uint32_t, int, bool) { return v; }
    __device__ static __forceinline__ T encode(R v) { return v; }
    __device__ static __forceinline__ R decode(T v) { return v; }
};

template <> struct Storage<LBM_F64> {
    using T = double;
    using R = double;
    static constexpr bool STOCHASTIC = false;
    static constexpr int SCALE_LOG2 = 0;
    __device__ static __forceinline__ R load(const T* p) { return *p; }
    __device__ static __forceinline__ R load_nc(const T* p) { return __ldg(p); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = v; }
    __device__ static __forceinline__ void store_sr(T* p, R v, uint32_t, int, bool) { *p = v; }
    __device__ static __forceinline__ R round(R v) { return v; }
    __device__ static __forceinline__ R round_sr(R v, uint32_t, int, bool) { return v; }
    __device__ static __forceinline__ T encode(R v) { return v; }
    __device__ static __forceinline__ R decode(T v) { return v; }
};

template <> struct Storage<LBM_F16> {
    using T = __half;
    using R = float;
    __device__ static __forceinline__ R decode(T v) { return __half2float(v) * FP16_INV_SCALE; }
    __device__ static __forceinline__ T encode(R v) { return __float2half_rn(v * FP16_SCALE); }
    // stochastic rounding of one value; hi: the odd node of its pair
    __device__ static __forceinline__ T encode_sr(R v, uint32_t h, int i, bool hi)
    {
        const float s = v * FP16_SCALE;
        const uint32_t w = cvt_rs_f16x2(s, s, sr_word(h, i));
        return __ushort_as_half((unsigned short)(hi ? w >> 16 : w));
    }
    static constexpr bool STOCHASTIC = true;
    __device__ static __forceinline__ R load(const T* p) { return decode(*p); }
    __device__ static __forceinline__ R load_nc(const T* p) { return decode(__ldg(p)); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = encode(v); }
    __device__ static __forceinline__ void store_sr(T* p, R v, uint32_t h, int i, bool hi) { *p = encode_sr(v, h, i, hi); }
    __device__ static __forceinline__ R round(R v) { return decode(encode(v)); }
    __device__ static __forceinline__ R round_sr(R v, uint32_t h, int i, bool hi) { return decode(encode_sr(v, h, i, hi)); }
    // The vector kernel computes on populations times 2^14 (collide with
    // SCALE_LOG2 = 14), so its conversions need no multiply.
    static constexpr int SCALE_LOG2 = 14;
    __device__ static __forceinline__ R decode_lo(uint32_t w) { return __low2float(*reinterpret_cast<const __half2*>(&w)); }
    __device__ static __forceinline__ R decode_hi(uint32_t w) { return __high2float(*reinterpret_cast<const __half2*>(&w)); }
    __device__ static __forceinline__ uint32_t pack_sr(R lo, R hi, uint32_t rbits) { return cvt_rs_f16x2(hi, lo, rbits); }
};

template <> struct Storage<LBM_BF16> {
    using T = __nv_bfloat16;
    using R = float;
    __device__ static __forceinline__ R decode(T v) { return __bfloat162float(v); }
    __device__ static __forceinline__ T encode(R v) { return __float2bfloat16_rn(v); }
    __device__ static __forceinline__ T encode_sr(R v, uint32_t h, int i, bool hi)
    {
        const uint32_t w = cvt_rs_bf16x2(v, v, sr_word(h, i));
        return __ushort_as_bfloat16((unsigned short)(hi ? w >> 16 : w));
    }
    static constexpr bool STOCHASTIC = true;
    __device__ static __forceinline__ R load(const T* p) { return decode(*p); }
    __device__ static __forceinline__ R load_nc(const T* p) { return decode(__ldg(p)); }
    __device__ static __forceinline__ void store(T* p, R v) { *p = encode(v); }
    __device__ static __forceinline__ void store_sr(T* p, R v, uint32_t h, int i, bool hi) { *p = encode_sr(v, h, i, hi); }
    __device__ static __forceinline__ R round(R v) { return decode(encode(v)); }
    __device__ static __forceinline__ R round_sr(R v, uint32_t h, int i, bool hi) { return decode(encode_sr(v, h, i, hi)); }
    static constexpr int SCALE_LOG2 = 0;
    __device__ static __forceinline__ R decode_lo(uint32_t w) { return __uint_as_float(w << 16); }
    __device__ static __forceinline__ R decode_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }
    __device__ static __forceinline__ uint32_t pack_sr(R lo, R hi, uint32_t rbits) { return cvt_rs_bf16x2(hi, lo, rbits); }
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
__device__ __forceinline__ float v_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double v_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float v_neg(float a) { return -a; }
__device__ __forceinline__ double v_neg(double a) { return -a; }
// Two nodes at once on the packed FP32x2 pipe (FFMA2/FADD2/FMUL2): each lane
// is the same IEEE operation as the scalar one, so a node pair updated this
// way gets the bits of two one-node updates, with half the instructions.
__device__ __forceinline__ float2 v_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 v_sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 v_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 v_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 v_rcp(float2 a) { return make_float2(__frcp_rn(a.x), __frcp_rn(a.y)); }
__device__ __forceinline__ float2 v_neg(float2 a) { return make_float2(-a.x, -a.y); }
// A scalar constant as a value of type V (both lanes for float2).
template <class V> struct Splat;
template <> struct Splat<float> { __device__ static __forceinline__ float of(float x) { return x; } };
template <> struct Splat<double> { __device__ static __forceinline__ double of(double x) { return x; } };
template <> struct Splat<float2> { __device__ static __forceinline__ float2 of(float x) { return make_float2(x, x); } };

// ---------------------------------------------------------------- collision
// TRT + Guo forcing on one node (reference src/lbm/collision.py:59-88,
// forcing.py:37-56). With rho = 1 + sum f~, u = (sum c f + F/2)/rho and, for
// each opposite pair (i, o = opp i), cu = c_i.u and cF = c_i.F, the update
//   f*_i = f_i - w+ (f+ - feq+) - w- (f- - feq-) + S+ + S-
// (f+- = (f_i +- f_o)/2, feq+ = w (drho + rho (4.5 cu^2 - 1.5 u.u)),
//  feq- = 3 w rho cu, S+ = w (1 - w+/2)(9 cu cF - 3 u.F), S- = 3 w (1 - w-/2) cF)
// is evaluated on the pair sums s = f_i + f_o and differences d = f_i - f_o,
// which also give the moments (drho = f_0 + sum s, j = sum c_i d):
//   P = hp s + E,  Qd = hm d + O,  f*_i = P + Qd,  f*_o = P - Qd
//   hp = (1 - w+)/2,  hm = (1 - w-)/2
//   E = (w A) + cu ((w B) cu + kC_i),  O = (w D) cu + kG_i
//   A = w+ (drho - 1.5 rho u.u) - 3 (1 - w+/2) u.F,  B = 4.5 w+ rho,  D = 3 w- rho
//   kC_i = (w 9 (1 - w+/2)) cF,  kG_i = (w 3 (1 - w-/2)) cF
// kC and kG depend on the force only: for a uniform force they are computed
// once per launch (relax_constants) and read as kernel parameters; w A, w B
// and w D once per weight. About 8 operations per pair; BGK is w- = w+. The
// rest population: f*_0 = (1 - w+) f_0 + w_0 A. One reciprocal per node.
// Every operation rounds explicitly (host and device alike), so all kernels,
// and constants computed on the host or per node, give the same bits.
//
// SCALE_LOG2 = k runs the update on populations multiplied by 2^k (float16
// storage keeps f~ 2^14 in its format): the moments are scaled back once and
// the weights and force terms carry 2^k. Scaling by a power of two is exact,
// so the result is 2^k times the unscaled one, bit for bit.
__host__ __device__ __forceinline__ float r_add(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ float r_sub(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ float r_mul(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ double r_add(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ double r_sub(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ double r_mul(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}

constexpr int QMAX = 19;

// Threads per block of the boundary-warp launches (LBM_LAUNCH_BOUNDARY).
constexpr int BOUNDARY_THREADS = 32;

// Default bound, in polls, of every wait of a TMA-staged kernel on an mbarrier.
constexpr uint32_t WAIT_LIMIT_DEFAULT = 1u << 22;

// Node-independent collision constants of one launch (see above).
template <class R>
struct Relax {
    R wp, one_m_wp, hp, hm, b45, d3, a3m;  // w+, 1 - w+, (1-w+)/2, (1-w-)/2, 4.5 w+, 3 w-, -3 (1 - w+/2)
    R c9, g3;                              // 9 (1 - w+/2), 3 (1 - w-/2)
    R kc[QMAX], kg[QMAX];                  // kC_i, kG_i of the uniform force
    R kcs[QMAX], kgs[QMAX];                // the same times 2^14 (float16 storage)
};

// c_i . F as a sum of +-components in x, y, z order (0 - F for a negative
// leading component, so a zero force gives +0 everywhere).
template <class L, class R>
__host__ __device__ __forceinline__ R guo_cf(int i, R Fx, R Fy, R Fz)
{
    R cF = R(0);
    bool first = true;
    if (L::cx(i) != 0) {
        cF = L::cx(i) > 0 ? Fx : r_sub(R(0), Fx);
        first = false;
    }
    if (L::cy(i) != 0) {
        if (first) cF = L::cy(i) > 0 ? Fy : r_sub(R(0), Fy);
        else cF = L::cy(i) > 0 ? r_add(cF, Fy) : r_sub(cF, Fy);
        first = false;
    }
    if (L::D == 3 && L::cz(i) != 0) {
        if (first) cF = L::cz(i) > 0 ? Fz : r_sub(R(0), Fz);
        else cF = L::cz(i) > 0 ? r_add(cF, Fz) : r_sub(cF, Fz);
    }
    return cF;
}

template <class L, class R>
__host__ __device__ inline void relax_scalars(Relax<R>& r, double wp_d, double wm_d)
{
    const R wp = R(wp_d), wm = R(wm_d);
    r.wp = wp;
    r.one_m_wp = r_sub(R(1), wp);
    r.hp = r_mul(R(0.5), r.one_m_wp);
    r.hm = r_mul(R(0.5), r_sub(R(1), wm));
    r.b45 = r_mul(R(4.5), wp);
    r.d3 = r_mul(R(3), wm);
    const R ap = r_sub(R(1), r_mul(R(0.5), wp)), am = r_sub(R(1), r_mul(R(0.5), wm));
    r.a3m = r_mul(R(-3), ap);
    r.c9 = r_mul(R(9), ap);
    r.g3 = r_mul(R(3), am);
}

template <class L, class R>
__host__ __device__ inline void relax_constants(Relax<R>& r, double wp, double wm, double fx, double fy, double fz)
{
    relax_scalars<L, R>(r, wp, wm);
    for (int i = 0; i < QMAX; ++i) {
        R kc = R(0), kg = R(0);
        if (i < L::Q) {
            const R cF = guo_cf<L, R>(i, R(fx), R(fy), R(fz));
            kc = r_mul(r_mul(R(L::w(i)), r.c9), cF);
            kg = r_mul(r_mul(R(L::w(i)), r.g3), cF);
        }
        r.kc[i] = kc;
        r.kg[i] = kg;
        r.kcs[i] = r_mul(kc, R(16384));
        r.kgs[i] = r_mul(kg, R(16384));
    }
}

// Force terms of the collision: from the launch constants (uniform force) ...
template <class R, int SCALE_LOG2>
struct UniformGuo {
    const Relax<R>& r;
    __device__ __forceinline__ R kc(int i) const { return SCALE_LOG2 ? r.kcs[i] : r.kc[i]; }
    __device__ __forceinline__ R kg(int i) const { return SCALE_LOG2 ? r.kgs[i] : r.kg[i]; }
};
// ... or computed for this node's force (per-node force fields)
template <class L, class R, int SCALE_LOG2>
struct NodeGuo {
    const Relax<R>& r;
    R Fx, Fy, Fz;
    __device__ __forceinline__ R k(int i, R coef) const
    {
        const R v = r_mul(r_mul(R(L::w(i)), coef), guo_cf<L, R>(i, Fx, Fy, Fz));
        return SCALE_LOG2 ? r_mul(v, R(1 << SCALE_LOG2)) : v;
    }
    __device__ __forceinline__ R kc(int i) const { return k(i, r.c9); }
    __device__ __forceinline__ R kg(int i) const { return k(i, r.g3); }
};

// V: the value type -- R for one node, float2 for a node pair (R = float).
template <class L, class R, int SCALE_LOG2, class Guo, class V>
__device__ __forceinline__ void collide(V (&f)[L::Q], const Relax<R>& c, V Fx, V Fy, V Fz, const Guo& guo)
{
    using P = Splat<V>;
    constexpr double SC = (double)(1 << SCALE_LOG2);
    V s[L::Q], d[L::Q];
    V drho = f[0];
    V jx = P::of(R(0)), jy = P::of(R(0)), jz = P::of(R(0));
    bool fx = true, fy = true, fz = true;
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        const int o = L::opp(i);
        if (o < i) continue;
        s[i] = v_add(f[i], f[o]);
        d[i] = v_sub(f[i], f[o]);
        drho = v_add(drho, s[i]);
        // j = sum c_i d over pairs (c_o = -c_i)
        if (L::cx(i) != 0) { jx = fx ? (L::cx(i) > 0 ? d[i] : v_neg(d[i])) : (L::cx(i) > 0 ? v_add(jx, d[i]) : v_sub(jx, d[i])); fx = false; }
        if (L::cy(i) != 0) { jy = fy ? (L::cy(i) > 0 ? d[i] : v_neg(d[i])) : (L::cy(i) > 0 ? v_add(jy, d[i]) : v_sub(jy, d[i])); fy = false; }
        if (L::D == 3 && L::cz(i) != 0) { jz = fz ? (L::cz(i) > 0 ? d[i] : v_neg(d[i])) : (L::cz(i) > 0 ? v_add(jz, d[i]) : v_sub(jz, d[i])); fz = false; }
    }
    if (SCALE_LOG2) {
        const V inv_sc = P::of(R(1.0 / SC));
        drho = v_mul(drho, inv_sc);
        jx = v_mul(jx, inv_sc);
        jy = v_mul(jy, inv_sc);
        if (L::D == 3) jz = v_mul(jz, inv_sc);
    }
    const V half = P::of(R(0.5));
    const V rho = v_add(P::of(R(1)), drho);
    const V inv = v_rcp(rho);
    const V ux = v_mul(v_fma(half, Fx, jx), inv);
    const V uy = v_mul(v_fma(half, Fy, jy), inv);
    const V uz = L::D == 3 ? v_mul(v_fma(half, Fz, jz), inv) : P::of(R(0));
    V usq = v_mul(ux, ux);
    usq = v_fma(uy, uy, usq);
    if (L::D == 3) usq = v_fma(uz, uz, usq);
    V uF = v_mul(ux, Fx);
    uF = v_fma(uy, Fy, uF);
    if (L::D == 3) uF = v_fma(uz, Fz, uF);
    // A = w+ (drho - 1.5 rho usq) - 3 (1 - w+/2) uF
    const V A = v_fma(P::of(c.a3m), uF, v_mul(P::of(c.wp), v_fma(v_mul(P::of(R(-1.5)), rho), usq, drho)));
    const V B = v_mul(P::of(c.b45), rho);
    const V Dm = v_mul(P::of(c.d3), rho);
    f[0] = v_fma(P::of(c.one_m_wp), f[0], v_mul(P::of(R(L::w(0) * SC)), A));
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        const int o = L::opp(i);
        if (o < i) continue;
        const V wi = P::of(R(L::w(i) * SC));
        V cu = P::of(R(0));
        bool first = true;
        if (L::cx(i) != 0) { cu = L::cx(i) > 0 ? ux : v_neg(ux); first = false; }
        if (L::cy(i) != 0) { cu = first ? (L::cy(i) > 0 ? uy : v_neg(uy)) : (L::cy(i) > 0 ? v_add(cu, uy) : v_sub(cu, uy)); first = false; }
        if (L::D == 3 && L::cz(i) != 0) cu = first ? (L::cz(i) > 0 ? uz : v_neg(uz)) : (L::cz(i) > 0 ? v_add(cu, uz) : v_sub(cu, uz));
        const V E = v_fma(cu, v_fma(v_mul(wi, B), cu, P::of(guo.kc(i))), v_mul(wi, A));
        const V O = v_fma(v_mul(wi, Dm), cu, P::of(guo.kg(i)));
        const V Pp = v_fma(P::of(c.hp), s[i], E);
        const V Qd = v_fma(P::of(c.hm), d[i], O);
        f[i] = v_add(Pp, Qd);
        f[o] = v_sub(Pp, Qd);
    }
}

// A node pair (x even, x + 1) with the uniform force on the packed FP32x2
// pipe: fa, fb in, post-collision fa, fb out -- the bits of two one-node
// collisions.
template <class L, int SCALE_LOG2>
__device__ __forceinline__ void collide_pair(float (&fa)[L::Q], float (&fb)[L::Q], const Relax<float>& c, float Fx,
                                             float Fy, float Fz)
{
    float2 f[L::Q];
#pragma unroll
    for (int i = 0; i < L::Q; ++i) f[i] = make_float2(fa[i], fb[i]);
    collide<L, float, SCALE_LOG2>(f, c, make_float2(Fx, Fx), make_float2(Fy, Fy), make_float2(Fz, Fz),
                                  UniformGuo<float, SCALE_LOG2>{c});
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        fa[i] = f[i].x;
        fb[i] = f[i].y;
    }
}

// Collision of one node whose force is (Fx, Fy, Fz): the launch's force
// terms when that is the uniform force and they were precomputed, else per
// node.
template <class L, class R, int SCALE_LOG2 = 0>
__device__ __forceinline__ void collide_node(R (&f)[L::Q], const Relax<R>& c, bool uniform, R Fx, R Fy, R Fz)
{
    if (uniform)
        collide<L, R, SCALE_LOG2>(f, c, Fx, Fy, Fz, UniformGuo<R, SCALE_LOG2>{c});
    else
        collide<L, R, SCALE_LOG2>(f, c, Fx, Fy, Fz, NodeGuo<L, R, SCALE_LOG2>{c, Fx, Fy, Fz});
}

// ---------------------------------------------------------------- regularised collision
// Projective regularisation (J. Latt and B. Chopard, Math. Comput. Simul. 72
// (2006) 165-168; T. Krueger et al., The Lattice Boltzmann Method, Springer
// 2017, sec. 10.6.5): the non-equilibrium part f^neq = f - feq is replaced by
// its projection on the Hermite polynomials up to second order before it
// relaxes, which filters the higher-order (ghost) moments that destabilise
// BGK/TRT at low viscosity. With H_i = c_i c_i - I/3 and cs^2 = 1/3:
//   P(f^neq)_i = w_i [3 c_i . m1 + 4.5 H_i : Pi],  m1 = sum c f^neq,  Pi = sum c c f^neq
// Guo forcing: u = (j + F/2)/rho, so m1 = -F/2 exactly, and the odd part of
// the update, (1 - w-) P_odd + (1 - w-/2) 3 w c.F = 1.5 w c.F, does not depend
// on the odd rate. On shifted populations (f~ = f - w):
//   Pi = sum c c f~ - rho u u - drho I/3        (second-order feq moments are exact on D2Q9/D3Q19)
//   f*_i = feq~_i + 1.5 w_i c_i.F + (1 - w+) 4.5 w_i (c_i.Pi.c_i - tr Pi/3)
//          + (1 - w+/2) w_i (9 (c_i.u)(c_i.F) - 3 u.F)
// feq~_i = w_i [drho + rho (3 cu + 4.5 cu^2 - 1.5 u.u)]. Every operation rounds
// explicitly, as in collide(). Used with the one-node kernels (SCALE_LOG2 = 0).
template <class L, class R>
__device__ __forceinline__ R reg_dot(int i, R ax, R ay, R az)
{
    R v = R(0);
    bool first = true;
    if (L::cx(i) != 0) { v = L::cx(i) > 0 ? ax : v_neg(ax); first = false; }
    if (L::cy(i) != 0) { v = first ? (L::cy(i) > 0 ? ay : v_neg(ay)) : (L::cy(i) > 0 ? v_add(v, ay) : v_sub(v, ay)); first = false; }
    if (L::D == 3 && L::cz(i) != 0) v = first ? (L::cz(i) > 0 ? az : v_neg(az)) : (L::cz(i) > 0 ? v_add(v, az) : v_sub(v, az));
    return v;
}

template <class L, class R>
__device__ __forceinline__ void collide_regularized(R (&f)[L::Q], const Relax<R>& c, R Fx, R Fy, R Fz)
{
    // moments of the streamed populations: drho, j, sum c c f~
    R drho = f[0], jx = R(0), jy = R(0), jz = R(0);
    R sxx = R(0), syy = R(0), szz = R(0), sxy = R(0), sxz = R(0), syz = R(0);
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        drho = v_add(drho, f[i]);
        const int cx = L::cx(i), cy = L::cy(i), cz = L::cz(i);
        if (cx) { jx = cx > 0 ? v_add(jx, f[i]) : v_sub(jx, f[i]); sxx = v_add(sxx, f[i]); }
        if (cy) { jy = cy > 0 ? v_add(jy, f[i]) : v_sub(jy, f[i]); syy = v_add(syy, f[i]); }
        if (L::D == 3 && cz) { jz = cz > 0 ? v_add(jz, f[i]) : v_sub(jz, f[i]); szz = v_add(szz, f[i]); }
        if (cx && cy) sxy = cx * cy > 0 ? v_add(sxy, f[i]) : v_sub(sxy, f[i]);
        if (L::D == 3 && cx && cz) sxz = cx * cz > 0 ? v_add(sxz, f[i]) : v_sub(sxz, f[i]);
        if (L::D == 3 && cy && cz) syz = cy * cz > 0 ? v_add(syz, f[i]) : v_sub(syz, f[i]);
    }
    const R half = R(0.5);
    const R rho = v_add(R(1), drho);
    const R inv = v_rcp(rho);
    const R ux = v_mul(v_fma(half, Fx, jx), inv);
    const R uy = v_mul(v_fma(half, Fy, jy), inv);
    const R uz = L::D == 3 ? v_mul(v_fma(half, Fz, jz), inv) : R(0);
    R usq = v_mul(ux, ux);
    usq = v_fma(uy, uy, usq);
    if (L::D == 3) usq = v_fma(uz, uz, usq);
    R uF = v_mul(ux, Fx);
    uF = v_fma(uy, Fy, uF);
    if (L::D == 3) uF = v_fma(uz, Fz, uF);
    // Pi = S - rho u u - drho/3 I
    const R d3 = v_mul(drho, R(1.0 / 3.0));
    const R pxx = v_sub(v_sub(sxx, v_mul(v_mul(rho, ux), ux)), d3);
    const R pyy = v_sub(v_sub(syy, v_mul(v_mul(rho, uy), uy)), d3);
    const R pzz = L::D == 3 ? v_sub(v_sub(szz, v_mul(v_mul(rho, uz), uz)), d3) : R(0);
    const R pxy = v_sub(sxy, v_mul(v_mul(rho, ux), uy));
    const R pxz = L::D == 3 ? v_sub(sxz, v_mul(v_mul(rho, ux), uz)) : R(0);
    const R pyz = L::D == 3 ? v_sub(syz, v_mul(v_mul(rho, uy), uz)) : R(0);
    R tr3 = v_add(pxx, pyy);
    if (L::D == 3) tr3 = v_add(tr3, pzz);
    tr3 = v_mul(tr3, R(1.0 / 3.0));
    const R keep = c.one_m_wp;                        // 1 - w+
    const R src = v_sub(R(1), v_mul(R(0.5), c.wp));   // 1 - w+/2
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        const int cx = L::cx(i), cy = L::cy(i), cz = L::cz(i);
        const R w = R(L::w(i));
        const R cu = reg_dot<L, R>(i, ux, uy, uz);
        const R cF = reg_dot<L, R>(i, Fx, Fy, Fz);
        // c.Pi.c over the nonzero components of c (c_a^2 = 1)
        R cpc = R(0);
        if (cx) cpc = v_add(cpc, pxx);
        if (cy) cpc = v_add(cpc, pyy);
        if (L::D == 3 && cz) cpc = v_add(cpc, pzz);
        if (cx && cy) cpc = cx * cy > 0 ? v_fma(R(2), pxy, cpc) : v_fma(R(-2), pxy, cpc);
        if (L::D == 3 && cx && cz) cpc = cx * cz > 0 ? v_fma(R(2), pxz, cpc) : v_fma(R(-2), pxz, cpc);
        if (L::D == 3 && cy && cz) cpc = cy * cz > 0 ? v_fma(R(2), pyz, cpc) : v_fma(R(-2), pyz, cpc);
        const R qpi = v_sub(cpc, tr3);
        // feq~ = w (drho + rho (3 cu + 4.5 cu^2 - 1.5 usq))
        const R poly = v_fma(v_mul(R(4.5), cu), cu, v_fma(R(3), cu, v_mul(R(-1.5), usq)));
        R out = v_mul(w, v_fma(rho, poly, drho));
        out = v_fma(v_mul(R(1.5), w), cF, out);
        out = v_fma(v_mul(v_mul(R(4.5), w), keep), qpi, out);
        const R s_even = v_fma(v_mul(R(9), cu), cF, v_mul(R(-3), uF));
        out = v_fma(v_mul(w, src), s_even, out);
        f[i] = out;
    }
}

// ---------------------------------------------------------------- cumulant collision (D2Q9)
// The cumulant method (M. Geier, M. Schoenherr, A. Pasquali, M. Krafczyk,
// Comput. Math. Appl. 70 (2015) 507-547: central moments by the 'chimera'
// transformation, sec. 3; forcing by the half-force velocity shift, sec. 2.4)
// on the tensor-product lattice D2Q9, whose populations carry the moments
// (m, n), m, n <= 2. About u = (j + F/2)/rho: k20 - k02 and k11 relax with w+,
// k20 + k02 -> 2 rho/3, k21, k12 -> 0, the fourth-order cumulant
// k22/rho - (k20 k02 + 2 k11^2)/rho^2 -> 0, k10, k01 mirrored (the force).
// Evaluated in deviations only, so round-off stays at the scale of the
// shifted populations: k~ are the central moments of f~ = f - w (chimera along
// x, then y); those of the weights are M_m(u_x) M_n(u_y), M = (1, -u, 1/3 + u^2),
// and each post-collision moment is formed directly as its difference from the
// weights' one, p = k* - M M:
//   p00 = drho, p10 = 2 u_x - k~10, p01 = 2 u_y - k~01,
//   D* = (1 - w+) ((k~20 - k~02) + (u_x^2 - u_y^2)), k11* = (1 - w+) (k~11 + u_x u_y),
//   a = drho/3 + D*/2, b = drho/3 - D*/2, p20 = a - u_x^2, p02 = b - u_y^2, p11 = k11* - u_x u_y,
//   p21 = u_y (1/3 + u_x^2), p12 = u_x (1/3 + u_y^2),
//   p22 = (drho/9 + a b + 2 k11*^2)/rho - (u_x^2 + u_y^2)/3 - u_x^2 u_y^2,
// then the inverse chimera along y, then x. Plain rounded operations (no
// fused multiply-add) in the order of the oracle's restatement, so a step
// without boundaries gives the oracle's bits. Used with the one-node kernels
// (SCALE_LOG2 = 0).
template <class R>
__device__ __forceinline__ void chimera(R am, R a0, R ap, R u, R& k0, R& k1, R& k2)
{
    k0 = v_add(v_add(am, a0), ap);
    const R s = v_sub(ap, am);
    k1 = v_sub(s, v_mul(u, k0));
    k2 = v_add(v_sub(v_add(ap, am), v_mul(v_mul(R(2), u), s)), v_mul(v_mul(u, u), k0));
}

template <class R>
__device__ __forceinline__ void chimera_inverse(R k0, R k1, R k2, R u, R& am, R& a0, R& ap)
{
    const R s = v_add(k1, v_mul(u, k0));
    const R p = v_sub(v_add(k2, v_mul(v_mul(R(2), u), s)), v_mul(v_mul(u, u), k0));
    am = v_mul(R(0.5), v_sub(p, s));
    a0 = v_sub(k0, p);
    ap = v_mul(R(0.5), v_add(p, s));
}

// The D2Q9 slot of direction (cx, cy).
template <class L>
__host__ __device__ constexpr int slot_of(int cx, int cy)
{
    int k = 0;
    for (int i = 0; i < L::Q; ++i)
        if (L::cx(i) == cx && L::cy(i) == cy) k = i;
    return k;
}

template <class L, class R>
__device__ __forceinline__ void collide_cumulant(R (&f)[L::Q], const Relax<R>& c, R Fx, R Fy)
{
    static_assert(L::D == 2 && L::Q == 9, "the cumulant collision is built for D2Q9");
    R drho = f[0], jx = R(0), jy = R(0);
#pragma unroll
    for (int i = 1; i < L::Q; ++i) drho = v_add(drho, f[i]);
    // momentum over the directions in slot order, as the oracle sums it
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        if (L::cx(i)) jx = L::cx(i) > 0 ? v_add(jx, f[i]) : v_sub(jx, f[i]);
        if (L::cy(i)) jy = L::cy(i) > 0 ? v_add(jy, f[i]) : v_sub(jy, f[i]);
    }
    const R rho = v_add(R(1), drho);
    const R ux = v_div(v_add(jx, v_mul(R(0.5), Fx)), rho);
    const R uy = v_div(v_add(jy, v_mul(R(0.5), Fy)), rho);
    R t0[3], t1[3], t2[3];  // along x, per row cy = -1, 0, 1
#pragma unroll
    for (int r = 0; r < 3; ++r)
        chimera(f[slot_of<L>(-1, r - 1)], f[slot_of<L>(0, r - 1)], f[slot_of<L>(1, r - 1)], ux, t0[r], t1[r], t2[r]);
    R k[3][3];
    chimera(t0[0], t0[1], t0[2], uy, k[0][0], k[0][1], k[0][2]);
    chimera(t1[0], t1[1], t1[2], uy, k[1][0], k[1][1], k[1][2]);
    chimera(t2[0], t2[1], t2[2], uy, k[2][0], k[2][1], k[2][2]);
    const R third = R(1.0 / 3.0);
    const R uxx = v_mul(ux, ux), uyy = v_mul(uy, uy), uxy = v_mul(ux, uy);
    const R keep = v_sub(R(1), c.wp);
    const R dev = v_mul(keep, v_add(v_sub(k[2][0], k[0][2]), v_sub(uxx, uyy)));
    const R k11 = v_mul(keep, v_add(k[1][1], uxy));
    const R d3 = v_mul(drho, third);
    const R a = v_add(d3, v_mul(R(0.5), dev));
    const R b = v_sub(d3, v_mul(R(0.5), dev));
    const R x = v_add(v_add(v_mul(drho, R(1.0 / 9.0)), v_mul(a, b)), v_mul(R(2), v_mul(k11, k11)));
    const R p22 = v_sub(v_sub(v_div(x, rho), v_mul(v_add(uxx, uyy), third)), v_mul(uxx, uyy));
    const R p[3][3] = {{drho, v_sub(v_mul(R(2), uy), k[0][1]), v_sub(b, uyy)},
                       {v_sub(v_mul(R(2), ux), k[1][0]), v_sub(k11, uxy), v_mul(ux, v_add(third, uyy))},
                       {v_sub(a, uxx), v_mul(uy, v_add(third, uxx)), p22}};
    R q0[3], q1[3], q2[3];  // q_m[r]: moment m along x of row r
    chimera_inverse(p[0][0], p[0][1], p[0][2], uy, q0[0], q0[1], q0[2]);
    chimera_inverse(p[1][0], p[1][1], p[1][2], uy, q1[0], q1[1], q1[2]);
    chimera_inverse(p[2][0], p[2][1], p[2][2], uy, q2[0], q2[1], q2[2]);
#pragma unroll
    for (int r = 0; r < 3; ++r)
        chimera_inverse(q0[r], q1[r], q2[r], ux, f[slot_of<L>(-1, r - 1)], f[slot_of<L>(0, r - 1)],
                        f[slot_of<L>(1, r - 1)]);
}

// The node update of collision model CM (LBM_COLLIDE_*): TRT/BGK, regularised or cumulant.
template <class L, class R, int CM>
__device__ __forceinline__ void collide_model(R (&f)[L::Q], const Relax<R>& c, bool uniform, R Fx, R Fy, R Fz)
{
    if constexpr (CM == LBM_COLLIDE_REGULARIZED)
        collide_regularized<L, R>(f, c, Fx, Fy, Fz);
    else if constexpr (CM == LBM_COLLIDE_CUMULANT && L::D == 2)
        collide_cumulant<L, R>(f, c, Fx, Fy);
    else
        collide_node<L, R>(f, c, uniform, Fx, Fy, Fz);
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
    uint32_t wait_limit;  // polls of a TMA-staged block's wait for a tile (lbm_launch_t.tma_wait_limit)
    int collision;        // LBM_COLLIDE_* (the kernels are instantiated per model)
    // Health and mass epilogue of a checked step (lbm_launch_t.health; null words: off).
    int64_t* health_words;    // [0] first bad pitched node (atomicMin), [1] 1 if non-finite (atomicMax)
    double* health_partial;   // one float64 sum per block of the launch
    int64_t health_slot0;     // partial slot of this launch's first block
    void* readout_rho;        // checked step: rho and u of the nodes it updates (lbm_health_t.rho / .u)
    void* readout_u;
    lbm_special_t sp;
    bool guo_const;    // rf/rd hold kC, kG of the uniform force (else computed per node)
    Relax<float> rf;   // collision constants (float arithmetic)
    Relax<double> rd;  // the same for float64 storage
    template <class R> __device__ __forceinline__ const Relax<R>& relax() const
    {
        if constexpr (sizeof(R) == 8)
            return rd;
        else
            return rf;
    }
};

// ---------------------------------------------------------------- health epilogue
// On the step that ends a chunk of the run loop, the step kernels also check
// the state they store (reference Solver._check_health, src/lbm/solver.py:162-172):
// per updated fluid node drho = sum_i f~*_i of the stored (rounded) values in
// direction order, bad if non-finite or drho <= -1; and they sum f~* in
// float64 (the mass minus the fluid node count). Each thread accumulates the
// nodes it updates; health_block then folds the block into one partial sum
// (warp shuffles, then the warps in order: a fixed order) and the rare bad
// nodes into the two status words with atomics.
struct NodeHealth {
    double dm = 0.0;               // sum of stored f~* of this thread's nodes
    long long bad = 0x7fffffffffffffffLL;  // smallest bad pitched node
    bool nonfinite = false;
};

template <class L, class R>
__device__ __forceinline__ void health_node(NodeHealth& hl, int64_t nd, const R (&v)[L::Q])
{
    R drho = v[0];
    double dm = (double)v[0];
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        drho = v_add(drho, v[i]);
        dm += (double)v[i];
    }
    hl.dm += dm;
    const bool nf = !isfinite(drho);
    if (nf || drho <= R(-1)) hl.bad = nd < hl.bad ? nd : hl.bad;
    hl.nonfinite |= nf;
}

// rho and u of a node's post-collision populations v (shifted, direction
// order) with the force F the collision applied (reference
// macroscopic_from_post_collision, src/lbm/diagnostics.py:72-80):
// rho = 1 + sum v, u = (sum c v - F/2) / rho, each operation rounded once.
// The readout kernel and the readout fused into a checked step both call it,
// so they give the same bits.
template <class L, class R>
__device__ __forceinline__ void macro_node(const R (&v)[L::Q], R Fx, R Fy, R Fz, R& rho, R (&u)[3])
{
    R drho = v[0], jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        drho = v_add(drho, v[i]);
        if (L::cx(i)) jx = L::cx(i) > 0 ? v_add(jx, v[i]) : v_sub(jx, v[i]);
        if (L::cy(i)) jy = L::cy(i) > 0 ? v_add(jy, v[i]) : v_sub(jy, v[i]);
        if (L::D == 3 && L::cz(i)) jz = L::cz(i) > 0 ? v_add(jz, v[i]) : v_sub(jz, v[i]);
    }
    rho = v_add(R(1), drho);
    u[0] = v_div(v_sub(jx, v_mul(R(0.5), Fx)), rho);
    u[1] = v_div(v_sub(jy, v_mul(R(0.5), Fy)), rho);
    u[2] = L::D == 3 ? v_div(v_sub(jz, v_mul(R(0.5), Fz)), rho) : R(0);
}

template <class L, class R>
__device__ __forceinline__ void store_macro(const R (&v)[L::Q], R Fx, R Fy, R Fz, int64_t nd, int64_t qstride,
                                            R* __restrict__ rho_out, R* __restrict__ u_out)
{
    R rho, u[3];
    macro_node<L, R>(v, Fx, Fy, Fz, rho, u);
    rho_out[nd] = rho;
#pragma unroll
    for (int a = 0; a < L::D; ++a) u_out[a * qstride + nd] = u[a];
}

// Every thread of the block calls it once (blocks are whole warps).
__device__ __forceinline__ void health_block(const StepArgs& a, const NodeHealth& hl, int64_t block)
{
    __shared__ double warp_dm[32];
    if (hl.bad != 0x7fffffffffffffffLL) atomicMin((unsigned long long*)a.health_words, (unsigned long long)hl.bad);
    if (hl.nonfinite) atomicMax((unsigned long long*)(a.health_words + 1), 1ull);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    double x = hl.dm;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if ((tid & 31) == 0) warp_dm[tid >> 5] = x;
    __syncthreads();
    if (tid == 0) {
        double sum = 0.0;
        const int warps = (int)((blockDim.x * blockDim.y + 31) >> 5);
        for (int w = 0; w < warps; ++w) sum += warp_dm[w];
        a.health_partial[a.health_slot0 + block] = sum;
    }
}

// The bulk (or fused) launch of a step advances the step counter: one thread
// writes the other slot, which no thread of this step reads.
__device__ __forceinline__ void advance_seed(const StepArgs& a)
{
    if (a.seed != nullptr && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 &&
        threadIdx.y == 0)
        a.seed[a.parity ^ 1] = a.seed[a.parity] + 1u;
}

// ---------------------------------------------------------------- host
// Unique id of the calling thread's current CUDA context (cuCtxGetId, which
// never hands the same id to two contexts of one process), or 0 if there is
// no current context or the driver cannot say. Per-device state that the
// library caches -- a device symbol's address, a kernel attribute -- belongs
// to one context: after cudaDeviceReset the device gets a new context, the
// library's device code is loaded again and the cached state is stale, so
// such caches are keyed by this id as well as by the device number.
inline unsigned long long current_context_id()
{
    using GetCurrentFn = int (*)(void**);
    using GetIdFn = int (*)(void*, unsigned long long*);
    auto entry = [](const char* name) -> void* {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return p;
    };
    static GetCurrentFn get_current = reinterpret_cast<GetCurrentFn>(entry("cuCtxGetCurrent"));
    static GetIdFn get_id = reinterpret_cast<GetIdFn>(entry("cuCtxGetId"));
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_current == nullptr || get_id == nullptr || get_current(&ctx) != 0 || ctx == nullptr) return 0;
    if (get_id(ctx, &id) != 0) return 0;
    return id;
}

}  // namespace lbm
