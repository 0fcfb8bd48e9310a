// Kernels around the step: initial equilibrium, population export/import,
// node classification, macroscopic readout, divergence watchdog, affine
// gathers/reductions (force probes) and the AA rule-term export priming.
#include <climits>
#include <mutex>

#include "dispatch.cuh"

namespace lbm {

// Natural slot of f*_i(node) in a stored state (pull and post-even AA layouts).
template <class L>
__device__ __forceinline__ int natural_slot(int i, int layout) { return layout == LBM_LAYOUT_AA_ODD ? L::opp(i) : i; }

// Node coordinates of a pitched index; false for padding (x >= nx, or the
// tail of a plane padded beyond pitch * ny * nz).
__device__ __forceinline__ bool decode_node(const lbm_grid_t& g, int64_t nd, int& x, int& y, int& z)
{
    const int64_t row = nd / g.pitch;
    x = (int)(nd - row * g.pitch);
    y = (int)(row % g.ny);
    z = (int)(row / g.ny);
    return x < g.nx && z < g.nz;
}

// ---------------------------------------------------------------- init
// Shifted equilibrium (reference src/lbm/equilibrium.py:40-58). The velocity
// is shifted by F/(2 rho) in float64 and cast once, as the reference does.
template <class L, int ST>
__global__ void init_kernel(const lbm_grid_t g, const lbm_physics_t p, const double* __restrict__ rho_in,
                            const double* __restrict__ u_in, int layout, typename Storage<ST>::T* f)
{
    using R = typename Storage<ST>::R;
    const int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (nd >= g.qstride) return;
    int x, y, z;
    if (!decode_node(g, nd, x, y, z)) return;
    const int64_t qs = g.qstride;
    const double rho_d = rho_in[nd];
    const R* ff = (const R*)p.force_field;
    R uc[3] = {R(0), R(0), R(0)};
    for (int a = 0; a < L::D; ++a) {
        const double F = p.force[a] + (ff != nullptr ? (double)ff[a * qs + nd] : 0.0);
        uc[a] = (R)(u_in[a * qs + nd] + 0.5 * F / rho_d);
    }
    const R dr = (R)(rho_d - 1.0);
    const R ux = uc[0], uy = uc[1], uz = uc[2];
    const R rho = R(1) + dr;
    const R usq = R(1.5) * (ux * ux + uy * uy + uz * uz);
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        const R cu = R(3) * (R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz);
        const R feq = R(L::w(i)) * (dr + rho * (cu + R(0.5) * cu * cu - usq));
        Storage<ST>::store(f + natural_slot<L>(i, layout) * qs + nd, feq);
    }
}

template <class L, int ST>
int init_equilibrium(const lbm_grid_t& g, const lbm_physics_t& p, const double* rho, const double* u, int layout,
                     void* f, cudaStream_t s)
{
    using T = typename Storage<ST>::T;
    if (layout != LBM_LAYOUT_PULL && layout != LBM_LAYOUT_AA_ODD) return LBM_ERR_INVALID;
    init_kernel<L, ST><<<blocks_for(g.qstride, 256), 256, 0, s>>>(g, p, rho, u, layout, (T*)f);
    return launch_status();
}

// ---------------------------------------------------------------- unpack / pack
template <class L, int ST, bool PACK>
__global__ void convert_kernel(const lbm_grid_t g, typename Storage<ST>::T* f, typename Storage<ST>::R* nat, int layout)
{
    const int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (nd >= g.qstride) return;
    int x, y, z;
    if (!decode_node(g, nd, x, y, z)) return;
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        const int64_t slot = natural_slot<L>(i, layout) * g.qstride + nd;
        if (PACK)
            Storage<ST>::store(f + slot, nat[i * g.qstride + nd]);
        else
            nat[i * g.qstride + nd] = Storage<ST>::load(f + slot);
    }
}

template <class L, int ST>
int unpack(const lbm_grid_t& g, const void* f, int layout, void* out, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    using T = typename Storage<ST>::T;
    if (layout != LBM_LAYOUT_PULL && layout != LBM_LAYOUT_AA_ODD) return LBM_ERR_INVALID;
    convert_kernel<L, ST, false><<<blocks_for(g.qstride, 256), 256, 0, s>>>(g, (T*)f, (R*)out, layout);
    return launch_status();
}

template <class L, int ST>
int pack(const lbm_grid_t& g, const void* in, int layout, void* f, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    using T = typename Storage<ST>::T;
    if (layout != LBM_LAYOUT_PULL && layout != LBM_LAYOUT_AA_ODD) return LBM_ERR_INVALID;
    convert_kernel<L, ST, true><<<blocks_for(g.qstride, 256), 256, 0, s>>>(g, (T*)f, (R*)in, layout);
    return launch_status();
}

// ---------------------------------------------------------------- classify
template <class L>
__global__ void classify_kernel(const lbm_grid_t g, const uint8_t* __restrict__ solid, uint8_t* __restrict__ kind,
                                uint32_t* __restrict__ nbr)
{
    const int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (nd >= g.qstride) return;
    int x, y, z;
    if (!decode_node(g, nd, x, y, z)) {
        kind[nd] = KIND_SOLID;  // padding: never updated, never a neighbour
        if (nbr) nbr[nd] = 0;
        return;
    }
    uint32_t m = 0;
#pragma unroll
    for (int i = 1; i < L::Q; ++i) {
        const int sx = wrap(x - L::cx(i), g.nx), sy = wrap(y - L::cy(i), g.ny);
        const int sz = L::D == 3 ? wrap(z - L::cz(i), g.nz) : 0;
        if (solid[((int64_t)sz * g.ny + sy) * g.pitch + sx]) m |= 1u << i;
    }
    if (nbr) nbr[nd] = m;
    if (solid[nd]) {
        kind[nd] = KIND_SOLID;
        return;
    }
    const bool edge = x == 0 || x == g.nx - 1 || y == 0 || y == g.ny - 1 || (L::D == 3 && (z == 0 || z == g.nz - 1));
    kind[nd] = (m ? KIND_NEAR : KIND_FLUID) | (edge ? KIND_EDGE : KIND_FLUID);
}

__global__ void mark_special_kernel(const int64_t* __restrict__ nodes, int n, uint8_t* kind)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) kind[nodes[s]] |= KIND_SPECIAL;
}

template <class L, int ST>
int classify(const lbm_grid_t& g, const uint8_t* solid, const int64_t* special, int n_special, uint8_t* kind,
             uint32_t* nbr, cudaStream_t s)
{
    classify_kernel<L><<<blocks_for(g.qstride, 256), 256, 0, s>>>(g, solid, kind, nbr);
    if (n_special > 0) mark_special_kernel<<<blocks_for(n_special, 256), 256, 0, s>>>(special, n_special, kind);
    return launch_status();
}

// ---------------------------------------------------------------- macroscopic
// rho = 1 + sum f~*, u = (sum c f* - F/2)/rho (reference diagnostics.py:72-80).
// Over every node, or (list mode) over the immersed-boundary nodes with their
// local force added to F.
template <class L, int ST>
__global__ void macro_kernel(const lbm_grid_t g, const lbm_physics_t p, const uint8_t* __restrict__ kind,
                             const typename Storage<ST>::T* __restrict__ f, int layout,
                             const int64_t* __restrict__ list, const typename Storage<ST>::R* __restrict__ local,
                             int n_list, typename Storage<ST>::R* __restrict__ rho_out,
                             typename Storage<ST>::R* __restrict__ u_out)
{
    using R = typename Storage<ST>::R;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t nd = t;
    if (list != nullptr) {
        if (t >= n_list) return;
        nd = list[t];
    } else if (nd >= g.qstride) {
        return;
    }
    int x, y, z;
    if (!decode_node(g, nd, x, y, z)) return;
    const int64_t qs = g.qstride;
    if (kind[nd] & KIND_SOLID) {
        rho_out[nd] = R(1);
        for (int a = 0; a < L::D; ++a) u_out[a * qs + nd] = R(0);
        return;
    }
    R v[L::Q];
#pragma unroll
    for (int i = 0; i < L::Q; ++i) v[i] = Storage<ST>::load(f + natural_slot<L>(i, layout) * qs + nd);
    R F[3] = {R(p.force[0]), R(p.force[1]), R(p.force[2])};
    if (p.force_field != nullptr) {
        const R* ff = (const R*)p.force_field;
        for (int a = 0; a < L::D; ++a) F[a] += ff[a * qs + nd];
    }
    if (list != nullptr && local != nullptr) {
        for (int a = 0; a < L::D; ++a) F[a] += local[(int64_t)a * n_list + t];
    }
    store_macro<L, R>(v, F[0], F[1], F[2], nd, qs, rho_out, u_out);
}

template <class L, int ST>
int macroscopic(const lbm_grid_t& g, const lbm_physics_t& p, const uint8_t* kind, const void* f, int layout,
                const int64_t* local_nodes, const void* local_force, int n_local, void* rho, void* u, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    using T = typename Storage<ST>::T;
    if (layout != LBM_LAYOUT_PULL && layout != LBM_LAYOUT_AA_ODD) return LBM_ERR_INVALID;
    macro_kernel<L, ST><<<blocks_for(g.qstride, 256), 256, 0, s>>>(g, p, kind, (const T*)f, layout, nullptr, nullptr,
                                                                   0, (R*)rho, (R*)u);
    if (n_local > 0 && local_nodes != nullptr)
        macro_kernel<L, ST><<<blocks_for(n_local, 256), 256, 0, s>>>(g, p, kind, (const T*)f, layout, local_nodes,
                                                                     (const R*)local_force, n_local, (R*)rho, (R*)u);
    return launch_status();
}

// ---------------------------------------------------------------- watchdog
__global__ void health_reset_kernel(int64_t* out)
{
    out[0] = LLONG_MAX;
    out[1] = 0;
}

template <class L, int ST>
__global__ void health_kernel(const lbm_grid_t g, const uint8_t* __restrict__ kind,
                              const typename Storage<ST>::T* __restrict__ f, int64_t* out)
{
    using R = typename Storage<ST>::R;
    const int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool bad = false, nonfinite = false;
    if (nd < g.qstride && !(kind[nd] & KIND_SOLID)) {
        R drho = Storage<ST>::load(f + nd);
#pragma unroll
        for (int i = 1; i < L::Q; ++i) drho += Storage<ST>::load(f + i * g.qstride + nd);
        nonfinite = !isfinite(drho);
        bad = nonfinite || drho <= R(-1);
    }
    const unsigned any_bad = __ballot_sync(0xffffffffu, bad);
    const unsigned any_nf = __ballot_sync(0xffffffffu, nonfinite);
    if (any_bad && (threadIdx.x & 31) == (unsigned)(__ffs(any_bad) - 1))
        atomicMin((unsigned long long*)out, (unsigned long long)nd);
    if (any_nf && (threadIdx.x & 31) == 0) atomicMax((unsigned long long*)(out + 1), 1ull);
}

// Sum of the checked step's per-block partials in a fixed order: 1024
// threads each add a strided subset in index order (four independent
// accumulators, combined in order), then a fixed tree.
__global__ void __launch_bounds__(1024) health_finish_kernel(const double* __restrict__ partial, int64_t n,
                                                             double* __restrict__ out)
{
    __shared__ double sums[1024];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int64_t i = threadIdx.x;
    for (; i + 3 * 1024 < n; i += 4 * 1024) {
        s0 += partial[i];
        s1 += partial[i + 1024];
        s2 += partial[i + 2 * 1024];
        s3 += partial[i + 3 * 1024];
    }
    for (; i < n; i += 1024) s0 += partial[i];
    sums[threadIdx.x] = (s0 + s1) + (s2 + s3);
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sums[threadIdx.x] += sums[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sums[0];
}

template <class L, int ST>
int health(const lbm_grid_t& g, const uint8_t* kind, const void* f, int64_t* out, cudaStream_t s)
{
    using T = typename Storage<ST>::T;
    health_kernel<L, ST><<<blocks_for(g.qstride, 256), 256, 0, s>>>(g, kind, (const T*)f, out);
    return launch_status();
}

// ---------------------------------------------------------------- affine
template <int ST>
__device__ __forceinline__ double affine_row(const typename Storage<ST>::T* __restrict__ f, const int64_t* __restrict__ slots,
                                             const double* __restrict__ coeff, const double* __restrict__ constant,
                                             int64_t r, int n_terms)
{
    double v = constant[r];
    for (int t = 0; t < n_terms; ++t) {
        const int64_t k = r * n_terms + t;
        const double c = coeff[k];
        if (c != 0.0) v += c * (double)Storage<ST>::load(f + slots[k]);
    }
    return v;
}

template <int ST>
__global__ void affine_gather_kernel(const typename Storage<ST>::T* __restrict__ f, const int64_t* __restrict__ slots,
                                     const double* __restrict__ coeff, const double* __restrict__ constant,
                                     int64_t n_rows, int n_terms, double* __restrict__ values)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r < n_rows) values[r] = affine_row<ST>(f, slots, coeff, constant, r, n_terms);
}

// One value per thread, weighted by weight[r][a]; warp-shuffle + shared-memory
// block sums go to partial[block][a]; the last block to finish adds the
// partials in block order (deterministic) and re-arms the counter.
template <int ST>
__global__ void __launch_bounds__(256) affine_reduce_kernel(
    const typename Storage<ST>::T* __restrict__ f, const int64_t* __restrict__ slots, const double* __restrict__ coeff,
    const double* __restrict__ constant, const double* __restrict__ weight, int64_t n_rows, int n_terms, int d,
    double* partial, unsigned* counter, double* out)
{
    __shared__ double warp_sums[8][3];
    __shared__ bool last;
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double v = 0.0;
    if (r < n_rows) v = affine_row<ST>(f, slots, coeff, constant, r, n_terms);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int a = 0; a < d; ++a) {
        double x = r < n_rows ? v * weight[r * d + a] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if (lane == 0) warp_sums[warp][a] = x;
    }
    __syncthreads();
    if (threadIdx.x < d) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += warp_sums[w][threadIdx.x];
        partial[(int64_t)blockIdx.x * d + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last && threadIdx.x < d) {
        __threadfence();
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += ((volatile double*)partial)[(int64_t)b * d + threadIdx.x];
        out[threadIdx.x] = s;
    }
    if (last && threadIdx.x == 0) *counter = 0u;
}

// ---------------------------------------------------------------- AA exports
template <class L, int ST>
__global__ void export_prime_kernel(const lbm_special_t sp, int64_t qstride, const typename Storage<ST>::T* __restrict__ f,
                                    int layout, typename Storage<ST>::R* __restrict__ out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= sp.n_special) return;
    const uint32_t mask = sp.export_mask[s];
    if (!mask) return;
    const int64_t nd = sp.node[s];
    const int e0 = sp.export_first[s];
#pragma unroll
    for (int k = 0; k < L::Q; ++k)
        if ((mask >> k) & 1u)
            out[e0 + __popc(mask & ((1u << k) - 1u))] = Storage<ST>::load(f + natural_slot<L>(k, layout) * qstride + nd);
}

template <class L, int ST>
int export_prime(const lbm_grid_t& g, const lbm_special_t& sp, const void* f, int layout, void* out, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    using T = typename Storage<ST>::T;
    if (layout != LBM_LAYOUT_PULL && layout != LBM_LAYOUT_AA_ODD) return LBM_ERR_INVALID;
    if (sp.n_special <= 0 || sp.n_export <= 0) return LBM_OK;
    export_prime_kernel<L, ST><<<blocks_for(sp.n_special, 128), 128, 0, s>>>(sp, g.qstride, (const T*)f, layout, (R*)out);
    return launch_status();
}

}  // namespace lbm

using namespace lbm;

static bool grid_ok(const lbm_grid_t* g)
{
    if (g == nullptr) return false;
    if (g->lattice != LBM_D2Q9 && g->lattice != LBM_D3Q19) return false;
    if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || g->pitch < g->nx) return false;
    if (g->lattice == LBM_D2Q9 && g->nz != 1) return false;
    return g->qstride >= (int64_t)g->pitch * g->ny * g->nz;
}

extern "C" int lbm_init_equilibrium(const lbm_grid_t* g, const lbm_physics_t* p, const double* rho, const double* u,
                                    int32_t layout, void* f, lbm_stream_t stream)
{
    if (!grid_ok(g) || !p || !rho || !u || !f) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, init_equilibrium, *g, *p, rho, u, layout, f, (cudaStream_t)stream);
}

extern "C" int lbm_unpack(const lbm_grid_t* g, const void* f, int32_t layout, void* out, lbm_stream_t stream)
{
    if (!grid_ok(g) || !f || !out) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, unpack, *g, f, layout, out, (cudaStream_t)stream);
}

extern "C" int lbm_pack(const lbm_grid_t* g, const void* in, int32_t layout, void* f, lbm_stream_t stream)
{
    if (!grid_ok(g) || !f || !in) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, pack, *g, in, layout, f, (cudaStream_t)stream);
}

extern "C" int lbm_classify(const lbm_grid_t* g, const uint8_t* solid, const int64_t* special, int32_t n_special,
                            uint8_t* kind, uint32_t* solid_nbr, lbm_stream_t stream)
{
    if (!grid_ok(g) || !solid || !kind || n_special < 0 || (n_special > 0 && !special)) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, classify, *g, solid, special, n_special, kind, solid_nbr, (cudaStream_t)stream);
}

extern "C" int lbm_macroscopic(const lbm_grid_t* g, const lbm_physics_t* p, const uint8_t* kind, const void* f,
                               int32_t layout, const int64_t* local_nodes, const void* local_force, int32_t n_local,
                               void* rho, void* u, lbm_stream_t stream)
{
    if (!grid_ok(g) || !p || !kind || !f || !rho || !u || n_local < 0) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, macroscopic, *g, *p, kind, f, layout, local_nodes, local_force, n_local, rho,
                 u, (cudaStream_t)stream);
}

extern "C" int lbm_health_reset(int64_t* out, lbm_stream_t stream)
{
    if (!out) return LBM_ERR_INVALID;
    health_reset_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(out);
    return launch_status();
}

extern "C" int lbm_health_finish(const lbm_health_t* h, double* delta_mass, lbm_stream_t stream)
{
    if (!h || !h->partial || h->n_partial <= 0 || !delta_mass) return LBM_ERR_INVALID;
    health_finish_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(h->partial, h->n_partial, delta_mass);
    return launch_status();
}

extern "C" int lbm_health(const lbm_grid_t* g, const uint8_t* kind, const void* f, int64_t* out, lbm_stream_t stream)
{
    if (!grid_ok(g) || !kind || !f || !out) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, health, *g, kind, f, out, (cudaStream_t)stream);
}

template <int ST>
static int affine_gather_t(const void* f, const int64_t* slots, const double* coeff, const double* constant,
                           int64_t n_rows, int n_terms, double* values, cudaStream_t s)
{
    affine_gather_kernel<ST><<<blocks_for(n_rows, 256), 256, 0, s>>>((const typename Storage<ST>::T*)f, slots, coeff,
                                                                     constant, n_rows, n_terms, values);
    return launch_status();
}

extern "C" int lbm_affine_gather(int32_t storage, const void* f, const int64_t* slots, const double* coeff,
                                 const double* constant, int64_t n_rows, int32_t n_terms, double* values,
                                 lbm_stream_t stream)
{
    if (!f || n_rows < 0 || n_terms < 0 || (n_rows > 0 && (!slots || !coeff || !constant || !values)))
        return LBM_ERR_INVALID;
    if (n_rows == 0) return LBM_OK;
    cudaStream_t s = (cudaStream_t)stream;
    switch (storage) {
    case LBM_F32: return affine_gather_t<LBM_F32>(f, slots, coeff, constant, n_rows, n_terms, values, s);
    case LBM_F64: return affine_gather_t<LBM_F64>(f, slots, coeff, constant, n_rows, n_terms, values, s);
    case LBM_F16: return affine_gather_t<LBM_F16>(f, slots, coeff, constant, n_rows, n_terms, values, s);
    case LBM_BF16: return affine_gather_t<LBM_BF16>(f, slots, coeff, constant, n_rows, n_terms, values, s);
    default: return LBM_ERR_INVALID;
    }
}

template <int ST>
static int affine_reduce_t(const void* f, const int64_t* slots, const double* coeff, const double* constant,
                           const double* weight, int64_t n_rows, int n_terms, int d, double* partial,
                           uint32_t* counter, double* out, cudaStream_t s)
{
    affine_reduce_kernel<ST><<<blocks_for(n_rows, 256), 256, 0, s>>>((const typename Storage<ST>::T*)f, slots, coeff,
                                                                     constant, weight, n_rows, n_terms, d, partial,
                                                                     counter, out);
    return launch_status();
}

extern "C" int lbm_affine_reduce(int32_t storage, const void* f, const int64_t* slots, const double* coeff,
                                 const double* constant, const double* weight, int64_t n_rows, int32_t n_terms,
                                 int32_t d, double* partial, uint32_t* counter, double* out, lbm_stream_t stream)
{
    if (!f || n_rows <= 0 || n_terms < 0 || d < 1 || d > 3 || !slots || !coeff || !constant || !weight || !partial ||
        !counter || !out)
        return LBM_ERR_INVALID;
    if ((n_rows + 255) / 256 > 0x7fffffffLL) return LBM_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    switch (storage) {
    case LBM_F32: return affine_reduce_t<LBM_F32>(f, slots, coeff, constant, weight, n_rows, n_terms, d, partial, counter, out, s);
    case LBM_F64: return affine_reduce_t<LBM_F64>(f, slots, coeff, constant, weight, n_rows, n_terms, d, partial, counter, out, s);
    case LBM_F16: return affine_reduce_t<LBM_F16>(f, slots, coeff, constant, weight, n_rows, n_terms, d, partial, counter, out, s);
    case LBM_BF16: return affine_reduce_t<LBM_BF16>(f, slots, coeff, constant, weight, n_rows, n_terms, d, partial, counter, out, s);
    default: return LBM_ERR_INVALID;
    }
}

// ---------------------------------------------------------------- affine reduce, no allocation
// lbm_affine_reduce_static runs affine_reduce_kernel with its scratch in this
// fixed array instead of caller buffers: a 256-byte head whose first word is
// the block counter, then partial[block][a] for up to
// LBM_AFFINE_REDUCE_STATIC_MAX_ROWS rows (3 doubles per 256-row block).
// Size: 256 B + 4096 * 3 * 8 B = 96.25 KiB per device.
constexpr int64_t kStaticReduceBlocks = (LBM_AFFINE_REDUCE_STATIC_MAX_ROWS + 255) / 256;
constexpr int64_t kStaticReduceHead = 32;  // doubles: 256 bytes
static __device__ __align__(256) double g_reduce_scratch[kStaticReduceHead + kStaticReduceBlocks * 3];

// Device address of g_reduce_scratch, looked up once per device context (with
// that device current) and cached; the lookup may load this library's device
// code. The cache is keyed by the context's id: after cudaDeviceReset the
// device's new context holds a new copy of the array, whose address is looked
// up again on the first call made in it.
constexpr int kMaxDevices = 64;
static std::mutex g_scratch_mutex;
static double* g_scratch_ptr[kMaxDevices];
static unsigned long long g_scratch_ctx[kMaxDevices];

static int static_reduce_scratch(double** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return LBM_ERR_LAUNCH;
    if (dev < 0 || dev >= kMaxDevices) return LBM_ERR_UNSUPPORTED;
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_ptr[dev] == nullptr || ctx == 0 || ctx != g_scratch_ctx[dev]) {
        void* p = nullptr;
        // (creates the device's context if this thread has none yet)
        if (cudaGetSymbolAddress(&p, g_reduce_scratch) != cudaSuccess || p == nullptr) return LBM_ERR_LAUNCH;
        g_scratch_ptr[dev] = static_cast<double*>(p);
        g_scratch_ctx[dev] = current_context_id();
    }
    *out = g_scratch_ptr[dev];
    return LBM_OK;
}

extern "C" int lbm_affine_reduce_static(int32_t storage, const void* f, const int64_t* slots, const double* coeff,
                                        const double* constant, const double* weight, int64_t n_rows,
                                        int32_t n_terms, int32_t d, double* out, lbm_stream_t stream)
{
    if (!f || n_rows <= 0 || n_terms < 0 || d < 1 || d > 3 || !slots || !coeff || !constant || !weight || !out)
        return LBM_ERR_INVALID;
    if (storage < LBM_F32 || storage > LBM_BF16) return LBM_ERR_INVALID;
    if (n_rows > LBM_AFFINE_REDUCE_STATIC_MAX_ROWS) return LBM_ERR_TOO_LARGE;
    double* scratch = nullptr;
    const int status = static_reduce_scratch(&scratch);
    if (status != LBM_OK) return status;
    uint32_t* counter = reinterpret_cast<uint32_t*>(scratch);
    double* partial = scratch + kStaticReduceHead;
    cudaStream_t s = (cudaStream_t)stream;
    // The kernel's last block re-arms the counter; clearing it here as well
    // keeps a call correct whatever state an earlier failed launch left.
    if (cudaMemsetAsync(counter, 0, sizeof(uint32_t), s) != cudaSuccess) return LBM_ERR_LAUNCH;
    return lbm_affine_reduce(storage, f, slots, coeff, constant, weight, n_rows, n_terms, d, partial, counter, out,
                             stream);
}

extern "C" int lbm_export_prime(const lbm_grid_t* g, const lbm_special_t* sp, const void* f, int32_t layout,
                                void* export_out, lbm_stream_t stream)
{
    if (!grid_ok(g) || !sp || !f || (sp->n_export > 0 && !export_out)) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, export_prime, *g, *sp, f, layout, export_out, (cudaStream_t)stream);
}
