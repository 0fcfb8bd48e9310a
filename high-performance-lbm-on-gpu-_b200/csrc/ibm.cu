// Immersed boundary method, direct forcing with multi-direct iterations
// (reference src/lbm/ibm.py:189-214), as one moments kernel plus one kernel
// per iteration instead of ~10 array operations per iteration.
//
// moments   : per stencil node n, the streamed populations f_k(n) = f*_k(n - c_k)
//             (stencils are clear of walls, so no bounce-back) give
//             rho_n and u*_n = (j_n + F_uniform/2) / rho_n.
// iteration : node-centric and deterministic (no atomics). Node n walks its
//             CSR list of (marker l, weight w_ln); for each marker it forms
//               rho_l = sum_s w_ls rho_s
//               U_l   = sum_s w_ls (u*_s + F_in,s / (2 rho_s))
//               F_l   = 2 rho_l (0 - U_l) dA_l
//             and accumulates w_ln F_l in float64; F_out,n = F_in,n + sum.
//             The node at stencil position 0 of marker l also records F_l
//             for the body force. Markers are recomputed by each of their
//             3^d nodes, which is cheaper than a second launch per pass.
#include "dispatch.cuh"

namespace lbm {

template <class L, int ST>
__global__ void ibm_moments_kernel(const lbm_grid_t g, const lbm_physics_t p, const lbm_ibm_t ib,
                                   const typename Storage<ST>::T* __restrict__ f, int layout)
{
    using R = typename Storage<ST>::R;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ib.n_nodes) return;
    const int64_t nd = ib.node[n];
    const int64_t row = nd / g.pitch;
    const int x = (int)(nd - row * g.pitch), y = (int)(row % g.ny), z = (int)(row / g.ny);
    R drho = R(0), jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
    for (int k = 0; k < L::Q; ++k) {
        int64_t slot;
        if (layout == LBM_LAYOUT_AA_EVEN) {
            slot = (int64_t)k * g.qstride + nd;  // odd step already pushed f*_k(n - c_k) to (k, n)
        } else {
            const int sx = wrap(x - L::cx(k), g.nx), sy = wrap(y - L::cy(k), g.ny);
            const int sz = L::D == 3 ? wrap(z - L::cz(k), g.nz) : 0;
            const int64_t src = ((int64_t)sz * g.ny + sy) * g.pitch + sx;
            const int kk = layout == LBM_LAYOUT_AA_ODD ? L::opp(k) : k;
            slot = (int64_t)kk * g.qstride + src;
        }
        const R fk = Storage<ST>::load(f + slot);
        drho = k == 0 ? fk : drho + fk;
        if (L::cx(k) > 0) jx += fk;
        if (L::cx(k) < 0) jx -= fk;
        if (L::cy(k) > 0) jy += fk;
        if (L::cy(k) < 0) jy -= fk;
        if (L::cz(k) > 0) jz += fk;
        if (L::cz(k) < 0) jz -= fk;
    }
    const R rho = R(1) + drho;
    R* rho_out = (R*)ib.rho;
    R* us = (R*)ib.u_star;
    rho_out[n] = rho;
    us[n] = (jx + R(0.5) * R(p.force[0])) / rho;
    us[ib.n_nodes + n] = (jy + R(0.5) * R(p.force[1])) / rho;
    if (L::D == 3) us[2 * ib.n_nodes + n] = (jz + R(0.5) * R(p.force[2])) / rho;
}

template <class L, int ST>
__global__ void ibm_iteration_kernel(const lbm_ibm_t ib, int iteration, const typename Storage<ST>::R* __restrict__ fin,
                                     typename Storage<ST>::R* __restrict__ fout)
{
    using R = typename Storage<ST>::R;
    constexpr int D = L::D;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ib.n_nodes) return;
    const int nn = ib.n_nodes;
    const R* __restrict__ rho = (const R*)ib.rho;
    const R* __restrict__ us = (const R*)ib.u_star;
    const R* __restrict__ wgt = (const R*)ib.weight;
    const R* __restrict__ area = (const R*)ib.area;
    const R* __restrict__ invw = (const R*)ib.inv_weight;
    R* mf = (R*)ib.marker_force + (int64_t)iteration * D * ib.n_markers;
    double acc[D];
#pragma unroll
    for (int a = 0; a < D; ++a) acc[a] = 0.0;
    for (int p = ib.inv_start[n]; p < ib.inv_start[n + 1]; ++p) {
        const int l = ib.inv_marker[p];
        const int* st = ib.stencil + (int64_t)l * ib.stencil_size;
        const R* wl = wgt + (int64_t)l * ib.stencil_size;
        R rho_l = R(0);
        R U[D];
#pragma unroll
        for (int a = 0; a < D; ++a) U[a] = R(0);
        for (int s = 0; s < ib.stencil_size; ++s) {
            const int m = st[s];
            const R w = wl[s];
            const R rm = rho[m];
            rho_l += w * rm;
#pragma unroll
            for (int a = 0; a < D; ++a) {
                R u = us[a * nn + m];
                if (fin != nullptr) u += fin[a * nn + m] / (R(2) * rm);
                U[a] += w * u;
            }
        }
        const R wn = invw[p];
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const R Fl = R(2) * rho_l * (R(0) - U[a]) * area[l];
            acc[a] += (double)(wn * Fl);
            if (st[0] == n) mf[(int64_t)a * ib.n_markers + l] = Fl;
        }
    }
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const double base = fin != nullptr ? (double)fin[a * nn + n] : 0.0;
        fout[a * nn + n] = (R)(base + acc[a]);
    }
}

// Body force -sum over passes and markers, one block, fixed order.
template <class L, int ST>
__global__ void ibm_body_force_kernel(const lbm_ibm_t ib, int iterations, double* out)
{
    using R = typename Storage<ST>::R;
    __shared__ double part[256];
    const R* mf = (const R*)ib.marker_force;
    for (int a = 0; a < L::D; ++a) {
        double s = 0.0;
        for (int it = 0; it < iterations; ++it)
            for (int l = threadIdx.x; l < ib.n_markers; l += blockDim.x)
                s += (double)mf[((int64_t)it * L::D + a) * ib.n_markers + l];
        part[threadIdx.x] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int k = 0; k < (int)blockDim.x; ++k) t += part[k];
            out[a] = -t;
        }
        __syncthreads();
    }
}

template <class L, int ST>
int ibm_moments(const lbm_grid_t& g, const lbm_physics_t& p, const lbm_ibm_t& ib, const void* f, int layout, cudaStream_t s)
{
    if (ib.n_nodes <= 0) return LBM_OK;
    ibm_moments_kernel<L, ST><<<blocks_for(ib.n_nodes, 128), 128, 0, s>>>(g, p, ib, (const typename Storage<ST>::T*)f, layout);
    return launch_status();
}

template <class L, int ST>
int ibm_iteration(const lbm_grid_t& g, const lbm_ibm_t& ib, int iteration, const void* fin, void* fout, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    if (ib.n_nodes <= 0) return LBM_OK;
    ibm_iteration_kernel<L, ST><<<blocks_for(ib.n_nodes, 128), 128, 0, s>>>(ib, iteration, (const R*)fin, (R*)fout);
    return launch_status();
}

template <class L, int ST>
int ibm_body_force(const lbm_grid_t& g, const lbm_ibm_t& ib, int iterations, double* out, cudaStream_t s)
{
    ibm_body_force_kernel<L, ST><<<1, 256, 0, s>>>(ib, iterations, out);
    return launch_status();
}

}  // namespace lbm

using namespace lbm;

static bool ibm_ok(const lbm_grid_t* g, const lbm_ibm_t* ib)
{
    if (!g || !ib || ib->n_nodes < 0 || ib->n_markers < 0) return false;
    const int expect = g->lattice == LBM_D2Q9 ? 9 : 27;
    if (ib->n_nodes > 0 && (ib->stencil_size != expect || !ib->node || !ib->stencil || !ib->weight || !ib->area ||
                            !ib->inv_start || !ib->inv_marker || !ib->inv_weight || !ib->rho || !ib->u_star ||
                            !ib->marker_force))
        return false;
    return true;
}

extern "C" int lbm_ibm_moments(const lbm_grid_t* g, const lbm_physics_t* p, const lbm_ibm_t* ib, const void* f,
                               int32_t layout, lbm_stream_t stream)
{
    if (!ibm_ok(g, ib) || !p || !f) return LBM_ERR_INVALID;
    if (layout < LBM_LAYOUT_PULL || layout > LBM_LAYOUT_AA_EVEN) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, ibm_moments, *g, *p, *ib, f, layout, (cudaStream_t)stream);
}

extern "C" int lbm_ibm_iteration(const lbm_grid_t* g, const lbm_ibm_t* ib, int32_t iteration, const void* force_in,
                                 void* force_out, lbm_stream_t stream)
{
    if (!ibm_ok(g, ib) || !force_out || iteration < 0 || force_in == force_out) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, ibm_iteration, *g, *ib, iteration, force_in, force_out, (cudaStream_t)stream);
}

extern "C" int lbm_ibm_body_force(const lbm_grid_t* g, const lbm_ibm_t* ib, int32_t iterations, double* out,
                                  lbm_stream_t stream)
{
    if (!ibm_ok(g, ib) || !out || iterations < 1) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, ibm_body_force, *g, *ib, iterations, out, (cudaStream_t)stream);
}
