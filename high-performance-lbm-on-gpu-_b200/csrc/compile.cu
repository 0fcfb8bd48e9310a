// Device-side rule compiler: the geometry and link-rule tables that the host
// builders compute, built on the GPU from the solid mask and the body.
//
//   lbm_ball_voxelize      solid |= nodes inside a circle / sphere
//                          (reference src/lbm/geometry.py:140-144, Ball.contains :74-76)
//   lbm_ball_links_count   \  every link from a fluid node into the ball, grouped by
//   lbm_ball_links_write   /  direction j, nodes ascending, with the wall fraction q
//                          (reference geometry.py:174-206 wall_links, Ball.ray_fraction :78-87)
//   lbm_bouzidi_links      the Bouzidi rule of every link (reference link_rules.py:154-188)
//   lbm_compile_terms      slots of affine terms in a stored layout (reference
//                          link_rules.py:203-240), pitched for this library's buffers
//   lbm_zou_he_count       \  the Zou-He rules of an open inlet or outlet column
//   lbm_zou_he_write       /  (reference open_boundaries.py:96-186)
//
// Node positions are the integer coordinates (x, y[, z]); every floating-point
// operation is an explicitly rounded IEEE operation in the order the host
// (NumPy) code evaluates it -- a sum over the axes left to right, no fused
// multiply-add -- so the device tables equal the host builders' bit for bit.
#include "dispatch.cuh"

namespace lbm {

struct BallArgs {
    double cx, cy, cz, r2;  // centre and squared radius (the host's radius**2)
};

// |p - c|^2 <= R^2, summed over x, y[, z] in that order.
template <class L>
__device__ __forceinline__ bool ball_contains(const BallArgs& b, int x, int y, int z)
{
    const double ox = __dsub_rn((double)x, b.cx), oy = __dsub_rn((double)y, b.cy);
    double s = __dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy));
    if (L::D == 3) {
        const double oz = __dsub_rn((double)z, b.cz);
        s = __dadd_rn(s, __dmul_rn(oz, oz));
    }
    return s <= b.r2;
}

// First t in (0, 1] where (x, y, z) + t d meets the sphere, d = -c_j:
//   a = d.d, b = 2 (o.d), k = o.o - R^2, t = (-b - sqrt(max(b^2 - 4 a k, 0))) / (2 a),
// clipped to [DBL_MIN, 1].
template <class L>
__device__ __forceinline__ double ball_fraction(const BallArgs& bl, int x, int y, int z, int j)
{
    const double ox = __dsub_rn((double)x, bl.cx), oy = __dsub_rn((double)y, bl.cy);
    const double oz = L::D == 3 ? __dsub_rn((double)z, bl.cz) : 0.0;
    const double dx = -(double)L::cx(j), dy = -(double)L::cy(j), dz = -(double)L::cz(j);
    double a = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
    double od = __dadd_rn(__dmul_rn(ox, dx), __dmul_rn(oy, dy));
    double oo = __dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy));
    if (L::D == 3) {
        a = __dadd_rn(a, __dmul_rn(dz, dz));
        od = __dadd_rn(od, __dmul_rn(oz, dz));
        oo = __dadd_rn(oo, __dmul_rn(oz, oz));
    }
    const double b = __dmul_rn(2.0, od);
    const double k = __dsub_rn(oo, bl.r2);
    double disc = __dsub_rn(__dmul_rn(b, b), __dmul_rn(__dmul_rn(4.0, a), k));
    disc = disc > 0.0 ? disc : 0.0;  // max(disc, 0) (NaN never occurs: finite inputs)
    double t = __ddiv_rn(__dsub_rn(-b, __dsqrt_rn(disc)), __dmul_rn(2.0, a));
    const double tiny = 2.2250738585072014e-308;  // smallest normal double
    t = t < tiny ? tiny : t;
    return t > 1.0 ? 1.0 : t;
}

__device__ __forceinline__ bool node_coords(const lbm_grid_t& g, int64_t nd, int& x, int& y, int& z)
{
    const int64_t row = nd / g.pitch;
    x = (int)(nd - row * g.pitch);
    y = (int)(row % g.ny);
    z = (int)(row / g.ny);
    return x < g.nx && z < g.nz;
}

constexpr int COMPILE_THREADS = 256;

// ---------------------------------------------------------------- voxelize
template <class L>
__global__ void ball_voxelize_kernel(const lbm_grid_t g, const BallArgs b, uint8_t* __restrict__ solid)
{
    const int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int x, y, z;
    if (nd >= g.qstride || !node_coords(g, nd, x, y, z)) return;
    if (ball_contains<L>(b, x, y, z)) solid[nd] = 1;
}

// ---------------------------------------------------------------- wall links
// Bit j of the node's mask: x is fluid and x - c_j (periodic) is inside the ball.
template <class L>
__device__ __forceinline__ uint32_t link_mask(const lbm_grid_t& g, const BallArgs& b, const uint8_t* solid, int64_t nd,
                                              int& x, int& y, int& z)
{
    if (nd >= g.qstride || !node_coords(g, nd, x, y, z) || solid[nd]) return 0u;
    uint32_t m = 0u;
#pragma unroll
    for (int j = 1; j < L::Q; ++j) {
        const int sx = wrap(x - L::cx(j), g.nx), sy = wrap(y - L::cy(j), g.ny);
        const int sz = L::D == 3 ? wrap(z - L::cz(j), g.nz) : 0;
        if (ball_contains<L>(b, sx, sy, sz)) m |= 1u << j;
    }
    return m;
}

// Pass 1: per (direction, block) link counts into offs[j * blocks + block];
// offs[Q * blocks + 1] counts nodes inside the ball that are not solid.
template <class L>
__global__ void __launch_bounds__(COMPILE_THREADS) ball_links_count_kernel(const lbm_grid_t g, const BallArgs b,
                                                                           const uint8_t* __restrict__ solid,
                                                                           int64_t* __restrict__ offs)
{
    __shared__ int counts[L::Q];
    if (threadIdx.x < L::Q) counts[threadIdx.x] = 0;
    __syncthreads();
    const int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int x = 0, y = 0, z = 0;
    const uint32_t m = link_mask<L>(g, b, solid, nd, x, y, z);
    for (int j = 1; j < L::Q; ++j) {
        const unsigned vote = __ballot_sync(0xffffffffu, (m >> j) & 1u);
        if ((threadIdx.x & 31) == 0 && vote) atomicAdd(&counts[j], __popc(vote));
    }
    if (nd < g.qstride && node_coords(g, nd, x, y, z) && !solid[nd] && ball_contains<L>(b, x, y, z))
        atomicAdd((unsigned long long*)&offs[(int64_t)L::Q * gridDim.x + 1], 1ull);
    __syncthreads();
    if (threadIdx.x < L::Q) offs[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = counts[threadIdx.x];
}

// Exclusive scan of offs[0 .. n) in place, total into offs[n], in three
// launches over blocks of SCAN_BLOCK entries: each block's sum into
// sums[b]; one block scans those sums (exclusive, total into sums[nb]); each
// block scans its entries and adds its offset.
constexpr int SCAN_BLOCK = 1024;

__device__ __forceinline__ int64_t warp_inclusive_scan(int64_t v, int lane)
{
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int64_t u = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += u;
    }
    return v;
}

// Exclusive scan of one value per thread over a block of SCAN_BLOCK threads;
// the block's total into *total.
__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* total)
{
    __shared__ int64_t warp_sum[SCAN_BLOCK / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t inc = warp_inclusive_scan(v, lane);
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int64_t w = warp_sum[lane];
        const int64_t winc = warp_inclusive_scan(w, lane);
        warp_sum[lane] = winc - w;
        if (lane == 31) *total = winc;
    }
    __syncthreads();
    return warp_sum[warp] + inc - v;
}

__global__ void __launch_bounds__(SCAN_BLOCK) scan_sums_kernel(const int64_t* __restrict__ offs, int64_t n,
                                                              int64_t* __restrict__ sums)
{
    __shared__ int64_t total;
    const int64_t i = blockIdx.x * (int64_t)SCAN_BLOCK + threadIdx.x;
    block_exclusive_scan(i < n ? offs[i] : 0, &total);
    __syncthreads();
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One block over nb (<= any size) block sums: runs of SCAN_BLOCK carried in order.
__global__ void __launch_bounds__(SCAN_BLOCK) scan_spine_kernel(int64_t* __restrict__ sums, int64_t nb)
{
    __shared__ int64_t total;
    int64_t carry = 0;
    for (int64_t base = 0; base < nb; base += SCAN_BLOCK) {
        const int64_t i = base + threadIdx.x;
        const int64_t v = i < nb ? sums[i] : 0;
        const int64_t ex = block_exclusive_scan(v, &total);
        if (i < nb) sums[i] = carry + ex;
        __syncthreads();
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = carry;
}

__global__ void __launch_bounds__(SCAN_BLOCK) scan_apply_kernel(int64_t* __restrict__ offs, int64_t n,
                                                               const int64_t* __restrict__ sums, int64_t nb)
{
    __shared__ int64_t total;
    const int64_t i = blockIdx.x * (int64_t)SCAN_BLOCK + threadIdx.x;
    const int64_t ex = block_exclusive_scan(i < n ? offs[i] : 0, &total);
    if (i < n) offs[i] = sums[blockIdx.x] + ex;
    if (blockIdx.x == 0 && threadIdx.x == 0) offs[n] = sums[nb];
}

// Pass 2: the links of direction j of this block go to offs[j * blocks + block]
// onwards in node order: rank = links of j in earlier warps of the block plus
// earlier lanes of this warp.
template <class L>
__global__ void __launch_bounds__(COMPILE_THREADS) ball_links_write_kernel(
    const lbm_grid_t g, const BallArgs b, const uint8_t* __restrict__ solid, const int64_t* __restrict__ offs,
    int64_t* __restrict__ node_out, int32_t* __restrict__ dir_out, double* __restrict__ q_out)
{
    __shared__ int warp_counts[COMPILE_THREADS / 32][L::Q];
    const int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int x = 0, y = 0, z = 0;
    const uint32_t m = link_mask<L>(g, b, solid, nd, x, y, z);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned votes[L::Q];
#pragma unroll
    for (int j = 1; j < L::Q; ++j) {
        votes[j] = __ballot_sync(0xffffffffu, (m >> j) & 1u);
        if (lane == 0) warp_counts[warp][j] = __popc(votes[j]);
    }
    __syncthreads();
    if (!m) return;
    const int64_t flat = ((int64_t)z * g.ny + y) * g.nx + x;  // natural (unpitched) node index
#pragma unroll
    for (int j = 1; j < L::Q; ++j) {
        if (!((m >> j) & 1u)) continue;
        int64_t pos = offs[(int64_t)j * gridDim.x + blockIdx.x] + __popc(votes[j] & ((1u << lane) - 1u));
        for (int w = 0; w < warp; ++w) pos += warp_counts[w][j];
        node_out[pos] = flat;
        dir_out[pos] = j;
        q_out[pos] = ball_fraction<L>(b, x, y, z, j);
    }
}

// ---------------------------------------------------------------- Bouzidi rules
// Per link (x, j, q), i = opp(j): keep = !(q < 1/2 and x + c_j solid); terms
//   q <  1/2: (i, x) 2q,       (i, x + c_j) 1 - 2q
//   q >= 1/2: (i, x) 0.5/q,    (j, x)       1 - 0.5/q
template <class L>
__global__ void bouzidi_kernel(const lbm_grid_t g, const uint8_t* __restrict__ solid, int64_t n,
                               const int64_t* __restrict__ node, const int32_t* __restrict__ dir,
                               const double* __restrict__ q, uint8_t* __restrict__ keep, int64_t* __restrict__ tdir,
                               int64_t* __restrict__ tnode, double* __restrict__ coeff)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int64_t flat = node[r];
    const int j = dir[r];
    const int x = (int)(flat % g.nx);
    const int64_t row = flat / g.nx;
    const int y = (int)(row % g.ny), z = (int)(row / g.ny);
    const int i = L::opp(j);
    const int bx = wrap(x + L::cx(j), g.nx), by = wrap(y + L::cy(j), g.ny);
    const int bz = L::D == 3 ? wrap(z + L::cz(j), g.nz) : 0;
    const int64_t behind = ((int64_t)bz * g.ny + by) * g.nx + bx;
    const bool blocked = solid[((int64_t)bz * g.ny + by) * g.pitch + bx] != 0;
    const double qq = q[r];
    const bool near = qq < 0.5;
    keep[r] = !(near && blocked);
    tdir[2 * r] = i;
    tnode[2 * r] = flat;
    tdir[2 * r + 1] = near ? i : j;
    tnode[2 * r + 1] = near ? behind : flat;
    coeff[2 * r] = near ? __dmul_rn(2.0, qq) : __ddiv_rn(0.5, qq);
    coeff[2 * r + 1] = near ? __dsub_rn(1.0, __dmul_rn(2.0, qq)) : __dsub_rn(1.0, __ddiv_rn(0.5, qq));
}

// ---------------------------------------------------------------- slot compiler
// Term t reads f*_{k}(y) (natural node y); its slot in the stored layout, pitched:
//   PULL:    k * qstride + p(y)
//   AA_ODD:  opp(k) * qstride + p(y)
//   AA_EVEN: k * qstride + p(y + c_k), or opp(k) * qstride + p(y) if y + c_k is solid, in which
//            case the value was stored with the wall term 6 w_opp(k) (c_opp(k) . u_w) added: the
//            term's share of its correction, coeff * 6 w_k (c_k . u_w(y + c_k)), goes to extra[t]
//            (wall: float64 (d, qstride) pitched, or NULL for walls at rest).
template <class L>
__global__ void compile_terms_kernel(const lbm_grid_t g, int layout, const uint8_t* __restrict__ solid,
                                     const double* __restrict__ wall, int64_t n, const int64_t* __restrict__ dir,
                                     const int64_t* __restrict__ node, const double* __restrict__ coeff,
                                     int64_t* __restrict__ slot, double* __restrict__ extra)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int k = (int)dir[t];
    const int64_t flat = node[t];
    const int x = (int)(flat % g.nx);
    const int64_t row = flat / g.nx;
    const int y = (int)(row % g.ny), z = (int)(row / g.ny);
    const int64_t p = ((int64_t)z * g.ny + y) * g.pitch + x;
    double e = 0.0;
    int64_t s;
    if (layout == LBM_LAYOUT_PULL) {
        s = (int64_t)k * g.qstride + p;
    } else if (layout == LBM_LAYOUT_AA_ODD) {
        s = (int64_t)L::opp(k) * g.qstride + p;
    } else {
        int cx = 0, cy = 0, cz = 0;
#pragma unroll
        for (int i = 0; i < L::Q; ++i)
            if (i == k) { cx = L::cx(i); cy = L::cy(i); cz = L::cz(i); }
        const int dx = wrap(x + cx, g.nx), dy = wrap(y + cy, g.ny), dz = L::D == 3 ? wrap(z + cz, g.nz) : 0;
        const int64_t pd = ((int64_t)dz * g.ny + dy) * g.pitch + dx;
        if (solid[pd]) {
            s = (int64_t)L::opp(k) * g.qstride + p;
            if (wall != nullptr) {
                double cu = __dmul_rn((double)cx, wall[pd]);
                cu = __dadd_rn(cu, __dmul_rn((double)cy, wall[g.qstride + pd]));
                if (L::D == 3) cu = __dadd_rn(cu, __dmul_rn((double)cz, wall[2 * g.qstride + pd]));
                double wk = 0.0;
#pragma unroll
                for (int i = 0; i < L::Q; ++i)
                    if (i == k) wk = L::w(i);
                e = __dmul_rn(coeff[t], __dmul_rn(__dmul_rn(6.0, wk), cu));
            }
        } else {
            s = (int64_t)k * g.qstride + pd;
        }
    }
    slot[t] = s;
    if (extra != nullptr) extra[t] = e;
}

// ---------------------------------------------------------------- Zou-He rules
// The rules of one open column x = column of a channel whose x = 0 and
// x = nx - 1 layers are closed (reference open_boundaries.py:96-153, in the
// Hecht-Harting form): velocity inlet (sign +1, velocity given at the
// column) or density outlet (sign -1, rho_out). Node (x, y, z) of the column,
// cross-section index c = z * ny + y, gets one rule per unknown population j
// (sign * c_jx = +1, ascending j) when it is fluid and some unknown streams in
// from the open layer (x - c_j in the layer, periodic wrap). A rule is a
// coefficient row over the node's Q streamed populations s_k = f*_k(x - c_k),
// or f*_opp(k)(x) when x - c_k is solid; with S0 + 2 S- = sum_k known_k s_k
// (known_k = 1 for c_n = 0, 2 for c_n = -1):
//   f_j = s_opp(j) + 6 w_j (c_j . rho u) - sum_t c_jt N_t,
//   N_t = 1/2 sum_{c_n = 0} s_k c_kt - rho u_t / 3,
//   inlet: rho u_a = u_a (S0 + 2 S-) / (1 - sign u_x); outlet: rho u_x = sign rho_out - sign (S0 + 2 S-),
// plus the shifted-storage constant b - w_j + sum_k a_k w_k. Every value is
// formed in the host builder's order, each operation rounded once.
struct ZouHeArgs {
    int column, sign;
    int layer_x;             // x of the open layer
    const uint8_t* layer;    // (nz * ny) fluid nodes of the open layer, before it was closed
    const double* velocity;  // (d, nz * ny) prescribed velocity at the column; NULL: outlet at rho_out
    double rho_out;
};

template <class L>
__device__ __forceinline__ int lat_c(int k, int a)
{
    return a == 0 ? L::cx(k) : (a == 1 ? L::cy(k) : L::cz(k));
}

template <class L>
__device__ __forceinline__ double zh_known(int k, int sign)
{
    const int cn = sign * L::cx(k);
    return cn == 0 ? 1.0 : (cn == -1 ? 2.0 : 0.0);
}

// rho u_a as an affine form: coefficient of s_k, and constant.
template <class L>
__device__ __forceinline__ double zh_rho_u_coeff(const ZouHeArgs& z, const double* u, double denom, int a, int k)
{
    const double known = zh_known<L>(k, z.sign);
    if (z.velocity != nullptr) return __dmul_rn(__ddiv_rn(known, denom), u[a]);
    return a == 0 ? __dmul_rn((double)(-z.sign), known) : 0.0;
}
__device__ __forceinline__ double zh_rho_u_const(const ZouHeArgs& z, int a)
{
    return (z.velocity == nullptr && a == 0) ? __dmul_rn((double)z.sign, z.rho_out) : 0.0;
}

template <class L>
__device__ __forceinline__ bool zh_touches(const lbm_grid_t& g, const ZouHeArgs& z, const uint8_t* solid, int y, int zz)
{
    const int x = z.column;
    if (solid[((int64_t)zz * g.ny + y) * g.pitch + x]) return false;
    bool hit = false;
#pragma unroll
    for (int j = 1; j < L::Q; ++j) {
        if (z.sign * L::cx(j) != 1) continue;
        const int sx = wrap(x - L::cx(j), g.nx), sy = wrap(y - L::cy(j), g.ny);
        const int sz = L::D == 3 ? wrap(zz - L::cz(j), g.nz) : 0;
        hit = hit || (sx == z.layer_x && z.layer[(int64_t)sz * g.ny + sy] != 0);
    }
    return hit;
}

// Row of unknown j at cross-section node c: coefficients over s_k and the shifted constant.
template <class L>
__device__ __forceinline__ void zh_row(const ZouHeArgs& z, const double* u, double denom, int j, double (&cf)[L::Q],
                                       double& constant)
{
    constexpr int Q = L::Q, D = L::D;
#pragma unroll
    for (int k = 0; k < Q; ++k) cf[k] = k == L::opp(j) ? 1.0 : 0.0;
    double b = 0.0;
    const double wj = L::w(j);
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const int cja = lat_c<L>(j, a);
        if (cja == 0) continue;
        const double s6 = __dmul_rn(__dmul_rn(6.0, wj), (double)cja);
#pragma unroll
        for (int k = 0; k < Q; ++k) cf[k] = __dadd_rn(cf[k], __dmul_rn(s6, zh_rho_u_coeff<L>(z, u, denom, a, k)));
        b = __dadd_rn(b, __dmul_rn(s6, zh_rho_u_const(z, a)));
    }
#pragma unroll
    for (int t = 1; t < D; ++t) {
        const int cjt = lat_c<L>(j, t);
        if (cjt == 0) continue;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            const double zero_n = z.sign * L::cx(k) == 0 ? 1.0 : 0.0;
            const double tc = __dsub_rn(__dmul_rn(__dmul_rn(0.5, zero_n), (double)lat_c<L>(k, t)),
                                        __ddiv_rn(zh_rho_u_coeff<L>(z, u, denom, t, k), 3.0));
            cf[k] = __dsub_rn(cf[k], __dmul_rn((double)cjt, tc));
        }
        b = __dsub_rn(b, __dmul_rn((double)cjt, __ddiv_rn(-zh_rho_u_const(z, t), 3.0)));
    }
    double acc = __dmul_rn(cf[0], L::w(0));
#pragma unroll
    for (int k = 1; k < Q; ++k) acc = __dadd_rn(acc, __dmul_rn(cf[k], L::w(k)));
    constant = __dadd_rn(__dsub_rn(b, wj), acc);
}

// The velocity at cross-section node c (d values) and 1 - sign u_x.
template <class L>
__device__ __forceinline__ double zh_velocity(const lbm_grid_t& g, const ZouHeArgs& z, int64_t c, double (&u)[3])
{
    const int64_t n = (int64_t)g.ny * g.nz;
#pragma unroll
    for (int a = 0; a < 3; ++a) u[a] = (z.velocity != nullptr && a < L::D) ? z.velocity[a * n + c] : 0.0;
    return __dsub_rn(1.0, __dmul_rn((double)z.sign, u[0]));
}

// Pass 1: offs[c] = 1 where node c of the column gets rules; the largest
// number of non-zero coefficients of a rule into offs[n + 1] (atomic max).
template <class L>
__global__ void __launch_bounds__(COMPILE_THREADS) zou_he_count_kernel(const lbm_grid_t g, const ZouHeArgs z,
                                                                       const uint8_t* __restrict__ solid,
                                                                       int64_t* __restrict__ offs)
{
    const int64_t n = (int64_t)g.ny * g.nz;
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int flag = 0, width = 0;
    if (c < n) {
        const int y = (int)(c % g.ny), zz = (int)(c / g.ny);
        if (zh_touches<L>(g, z, solid, y, zz)) {
            flag = 1;
            double u[3];
            const double denom = zh_velocity<L>(g, z, c, u);
#pragma unroll
            for (int j = 1; j < L::Q; ++j) {
                if (z.sign * L::cx(j) != 1) continue;
                double cf[L::Q], b;
                zh_row<L>(z, u, denom, j, cf, b);
                int nz = 0;
#pragma unroll
                for (int k = 0; k < L::Q; ++k) nz += cf[k] != 0.0;
                width = max(width, nz);
            }
        }
        offs[c] = flag;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) width = max(width, __shfl_xor_sync(0xffffffffu, width, off));
    if ((threadIdx.x & 31) == 0 && width > 0) atomicMax((unsigned long long*)&offs[n + 1], (unsigned long long)width);
}

// Pass 2: node c's rules at rows offs[c] * n_unknown onwards (unknowns
// ascending), their non-zero terms packed to the front in ascending k, the
// rest of the width zero.
template <class L>
__global__ void __launch_bounds__(COMPILE_THREADS) zou_he_write_kernel(
    const lbm_grid_t g, const ZouHeArgs z, const uint8_t* __restrict__ solid, const int64_t* __restrict__ offs,
    int width, int64_t* __restrict__ node_out, int64_t* __restrict__ dir_out, int64_t* __restrict__ tdir,
    int64_t* __restrict__ tnode, double* __restrict__ coeff, double* __restrict__ constant)
{
    const int64_t n = (int64_t)g.ny * g.nz;
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int x = z.column, y = (int)(c % g.ny), zz = (int)(c / g.ny);
    if (!zh_touches<L>(g, z, solid, y, zz)) return;
    double u[3];
    const double denom = zh_velocity<L>(g, z, c, u);
    const int64_t flat = ((int64_t)zz * g.ny + y) * g.nx + x;
    // the streamed population s_k: (k, x - c_k), or (opp k, x) where x - c_k is solid
    int64_t key_node[L::Q];
    int key_dir[L::Q];
#pragma unroll
    for (int k = 0; k < L::Q; ++k) {
        const int sx = wrap(x - L::cx(k), g.nx), sy = wrap(y - L::cy(k), g.ny);
        const int sz = L::D == 3 ? wrap(zz - L::cz(k), g.nz) : 0;
        const bool blocked = solid[((int64_t)sz * g.ny + sy) * g.pitch + sx] != 0;
        key_dir[k] = blocked ? L::opp(k) : k;
        key_node[k] = blocked ? flat : ((int64_t)sz * g.ny + sy) * g.nx + sx;
    }
    int n_unknown = 0;
#pragma unroll
    for (int j = 1; j < L::Q; ++j) n_unknown += z.sign * L::cx(j) == 1;
    int64_t row = offs[c] * n_unknown;
#pragma unroll
    for (int j = 1; j < L::Q; ++j) {
        if (z.sign * L::cx(j) != 1) continue;
        double cf[L::Q], b;
        zh_row<L>(z, u, denom, j, cf, b);
        node_out[row] = flat;
        dir_out[row] = j;
        constant[row] = b;
        int p = 0;
#pragma unroll
        for (int k = 0; k < L::Q; ++k) {
            if (cf[k] == 0.0 || p >= width) continue;
            tdir[row * width + p] = key_dir[k];
            tnode[row * width + p] = key_node[k];
            coeff[row * width + p] = cf[k];
            ++p;
        }
        for (; p < width; ++p) {
            tdir[row * width + p] = 0;
            tnode[row * width + p] = 0;
            coeff[row * width + p] = 0.0;
        }
        ++row;
    }
}

template <class L, int ST>
int zou_he_count(const lbm_grid_t& g, const ZouHeArgs& z, const uint8_t* solid, int64_t* offs, cudaStream_t s)
{
    const int64_t n = (int64_t)g.ny * g.nz;
    const int64_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    int64_t* sums = offs + n + 2;
    if (cudaMemsetAsync(offs + n + 1, 0, sizeof(int64_t), s) != cudaSuccess) return LBM_ERR_LAUNCH;
    zou_he_count_kernel<L><<<blocks_for(n, COMPILE_THREADS), COMPILE_THREADS, 0, s>>>(g, z, solid, offs);
    scan_sums_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(offs, n, sums);
    scan_spine_kernel<<<1, SCAN_BLOCK, 0, s>>>(sums, nb);
    scan_apply_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(offs, n, sums, nb);
    return launch_status();
}

template <class L, int ST>
int zou_he_write(const lbm_grid_t& g, const ZouHeArgs& z, const uint8_t* solid, const int64_t* offs, int width,
                 int64_t* node, int64_t* dir, int64_t* tdir, int64_t* tnode, double* coeff, double* constant,
                 cudaStream_t s)
{
    const int64_t n = (int64_t)g.ny * g.nz;
    zou_he_write_kernel<L><<<blocks_for(n, COMPILE_THREADS), COMPILE_THREADS, 0, s>>>(g, z, solid, offs, width, node,
                                                                                     dir, tdir, tnode, coeff, constant);
    return launch_status();
}

template <class L, int ST>
int ball_voxelize(const lbm_grid_t& g, BallArgs b, uint8_t* solid, cudaStream_t s)
{
    ball_voxelize_kernel<L><<<blocks_for(g.qstride, COMPILE_THREADS), COMPILE_THREADS, 0, s>>>(g, b, solid);
    return launch_status();
}

inline unsigned link_blocks(const lbm_grid_t& g) { return blocks_for(g.qstride, COMPILE_THREADS); }

template <class L, int ST>
int ball_links_count(const lbm_grid_t& g, BallArgs b, const uint8_t* solid, int64_t* offs, cudaStream_t s)
{
    const unsigned blocks = link_blocks(g);
    const int64_t n = (int64_t)L::Q * blocks;
    const int64_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    int64_t* sums = offs + n + 2;  // nb + 1 entries after the two result words
    if (cudaMemsetAsync(offs + n + 1, 0, sizeof(int64_t), s) != cudaSuccess) return LBM_ERR_LAUNCH;
    ball_links_count_kernel<L><<<blocks, COMPILE_THREADS, 0, s>>>(g, b, solid, offs);
    scan_sums_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(offs, n, sums);
    scan_spine_kernel<<<1, SCAN_BLOCK, 0, s>>>(sums, nb);
    scan_apply_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(offs, n, sums, nb);
    return launch_status();
}

template <class L, int ST>
int ball_links_write(const lbm_grid_t& g, BallArgs b, const uint8_t* solid, const int64_t* offs, int64_t* node,
                     int32_t* dir, double* q, cudaStream_t s)
{
    ball_links_write_kernel<L><<<link_blocks(g), COMPILE_THREADS, 0, s>>>(g, b, solid, offs, node, dir, q);
    return launch_status();
}

template <class L, int ST>
int bouzidi_links(const lbm_grid_t& g, const uint8_t* solid, int64_t n, const int64_t* node, const int32_t* dir,
                  const double* q, uint8_t* keep, int64_t* tdir, int64_t* tnode, double* coeff, cudaStream_t s)
{
    if (n == 0) return LBM_OK;
    bouzidi_kernel<L><<<blocks_for(n, COMPILE_THREADS), COMPILE_THREADS, 0, s>>>(g, solid, n, node, dir, q, keep,
                                                                                tdir, tnode, coeff);
    return launch_status();
}

template <class L, int ST>
int compile_terms(const lbm_grid_t& g, int layout, const uint8_t* solid, const double* wall, int64_t n,
                  const int64_t* dir, const int64_t* node, const double* coeff, int64_t* slot, double* extra,
                  cudaStream_t s)
{
    if (n == 0) return LBM_OK;
    compile_terms_kernel<L><<<blocks_for(n, COMPILE_THREADS), COMPILE_THREADS, 0, s>>>(g, layout, solid, wall, n, dir,
                                                                                      node, coeff, slot, extra);
    return launch_status();
}

}  // namespace lbm

using namespace lbm;

static bool compile_grid_ok(const lbm_grid_t* g)
{
    if (g == nullptr) return false;
    if (g->lattice != LBM_D2Q9 && g->lattice != LBM_D3Q19) return false;
    if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || g->pitch < g->nx) return false;
    if (g->lattice == LBM_D2Q9 && g->nz != 1) return false;
    return g->qstride >= (int64_t)g->pitch * g->ny * g->nz;
}

static int lattice_q(int lattice) { return lattice == LBM_D2Q9 ? 9 : 19; }

extern "C" int64_t lbm_ball_links_scratch(const lbm_grid_t* g)
{
    if (!compile_grid_ok(g)) return LBM_ERR_INVALID;
    const int64_t n = (int64_t)lattice_q(g->lattice) * link_blocks(*g);
    return n + 2 + (n + SCAN_BLOCK - 1) / SCAN_BLOCK + 1;  // counts, two result words, the scan's block sums
}

extern "C" int lbm_ball_voxelize(const lbm_grid_t* g, double cx, double cy, double cz, double radius_sq, uint8_t* solid,
                                 lbm_stream_t stream)
{
    if (!compile_grid_ok(g) || !solid || !(radius_sq > 0.0)) return LBM_ERR_INVALID;
    const BallArgs b{cx, cy, cz, radius_sq};
    LBM_DISPATCH(g->lattice, LBM_F64, ball_voxelize, *g, b, solid, (cudaStream_t)stream);
}

extern "C" int lbm_ball_links_count(const lbm_grid_t* g, const uint8_t* solid, double cx, double cy, double cz,
                                    double radius_sq, int64_t* scratch, lbm_stream_t stream)
{
    if (!compile_grid_ok(g) || !solid || !scratch || !(radius_sq > 0.0)) return LBM_ERR_INVALID;
    const BallArgs b{cx, cy, cz, radius_sq};
    LBM_DISPATCH(g->lattice, LBM_F64, ball_links_count, *g, b, solid, scratch, (cudaStream_t)stream);
}

extern "C" int lbm_ball_links_write(const lbm_grid_t* g, const uint8_t* solid, double cx, double cy, double cz,
                                    double radius_sq, const int64_t* scratch, int64_t* node, int32_t* direction,
                                    double* q, lbm_stream_t stream)
{
    if (!compile_grid_ok(g) || !solid || !scratch || !node || !direction || !q || !(radius_sq > 0.0))
        return LBM_ERR_INVALID;
    const BallArgs b{cx, cy, cz, radius_sq};
    LBM_DISPATCH(g->lattice, LBM_F64, ball_links_write, *g, b, solid, scratch, node, direction, q, (cudaStream_t)stream);
}

extern "C" int lbm_bouzidi_links(const lbm_grid_t* g, const uint8_t* solid, int64_t n, const int64_t* node,
                                 const int32_t* direction, const double* q, uint8_t* keep, int64_t* term_dir,
                                 int64_t* term_node, double* coeff, lbm_stream_t stream)
{
    if (!compile_grid_ok(g) || !solid || n < 0) return LBM_ERR_INVALID;
    if (n > 0 && (!node || !direction || !q || !keep || !term_dir || !term_node || !coeff)) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, LBM_F64, bouzidi_links, *g, solid, n, node, direction, q, keep, term_dir, term_node, coeff,
                 (cudaStream_t)stream);
}

extern "C" int lbm_compile_terms(const lbm_grid_t* g, int32_t layout, const uint8_t* solid, const double* wall_u,
                                 int64_t n, const int64_t* direction, const int64_t* node, const double* coeff,
                                 int64_t* slot, double* extra, lbm_stream_t stream)
{
    if (!compile_grid_ok(g) || n < 0) return LBM_ERR_INVALID;
    if (layout != LBM_LAYOUT_PULL && layout != LBM_LAYOUT_AA_ODD && layout != LBM_LAYOUT_AA_EVEN) return LBM_ERR_INVALID;
    if (n > 0 && (!direction || !node || !slot)) return LBM_ERR_INVALID;
    if (layout == LBM_LAYOUT_AA_EVEN && n > 0 && (!solid || (wall_u && (!coeff || !extra)))) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, LBM_F64, compile_terms, *g, layout, solid, wall_u, n, direction, node, coeff, slot, extra,
                 (cudaStream_t)stream);
}

// An inlet (sign +1) takes its velocity field, an outlet (sign -1) none.
static bool zou_he_ok(const lbm_grid_t* g, const uint8_t* solid, int32_t column, int32_t sign, int32_t layer_x,
                      const uint8_t* layer, const double* velocity)
{
    if (!compile_grid_ok(g) || !solid || !layer || (sign != 1 && sign != -1)) return false;
    if ((sign == 1) != (velocity != nullptr)) return false;
    return column >= 0 && column < g->nx && layer_x >= 0 && layer_x < g->nx;
}

extern "C" int64_t lbm_zou_he_scratch(const lbm_grid_t* g)
{
    if (!compile_grid_ok(g)) return LBM_ERR_INVALID;
    const int64_t n = (int64_t)g->ny * g->nz;
    return n + 2 + (n + SCAN_BLOCK - 1) / SCAN_BLOCK + 1;  // flags, two result words, the scan's block sums
}

extern "C" int lbm_zou_he_count(const lbm_grid_t* g, const uint8_t* solid, int32_t column, int32_t sign,
                                int32_t layer_x, const uint8_t* layer, const double* velocity, double rho_out,
                                int64_t* scratch, lbm_stream_t stream)
{
    if (!zou_he_ok(g, solid, column, sign, layer_x, layer, velocity) || !scratch) return LBM_ERR_INVALID;
    const ZouHeArgs z{column, sign, layer_x, layer, velocity, rho_out};
    LBM_DISPATCH(g->lattice, LBM_F64, zou_he_count, *g, z, solid, scratch, (cudaStream_t)stream);
}

extern "C" int lbm_zou_he_write(const lbm_grid_t* g, const uint8_t* solid, int32_t column, int32_t sign,
                                int32_t layer_x, const uint8_t* layer, const double* velocity, double rho_out,
                                const int64_t* scratch, int32_t width, int64_t* node, int64_t* direction,
                                int64_t* term_dir, int64_t* term_node, double* coeff, double* constant,
                                lbm_stream_t stream)
{
    if (!zou_he_ok(g, solid, column, sign, layer_x, layer, velocity) || !scratch || width < 1) return LBM_ERR_INVALID;
    if (!node || !direction || !term_dir || !term_node || !coeff || !constant) return LBM_ERR_INVALID;
    const ZouHeArgs z{column, sign, layer_x, layer, velocity, rho_out};
    LBM_DISPATCH(g->lattice, LBM_F64, zou_he_write, *g, z, solid, scratch, width, node, direction, term_dir, term_node,
                 coeff, constant, (cudaStream_t)stream);
}
