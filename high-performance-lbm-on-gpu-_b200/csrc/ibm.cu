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
#include "step_kernels.cuh"

namespace lbm {

template <class L, int ST>
__device__ __forceinline__ void ibm_moments_node(const lbm_grid_t& g, const lbm_physics_t& p, const lbm_ibm_t& ib,
                                                 const typename Storage<ST>::T* __restrict__ f, int layout, int n,
                                                 typename Storage<ST>::R* s_rho = nullptr,
                                                 typename Storage<ST>::R* s_us = nullptr, int64_t nd_loaded = -1)
{
    using R = typename Storage<ST>::R;
    const int64_t nd = nd_loaded >= 0 ? nd_loaded : ib.node[n];
    int x, y, z;
    if (g.qstride <= 0x7fffffffLL) {  // 32-bit index arithmetic (a 64-bit division is a long subroutine)
        const int row = (int)nd / g.pitch;
        x = (int)nd - row * g.pitch;
        y = row % g.ny;
        z = row / g.ny;
    } else {
        const int64_t row = nd / g.pitch;
        x = (int)(nd - row * g.pitch);
        y = (int)(row % g.ny);
        z = (int)(row / g.ny);
    }
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
    const R u[3] = {(jx + R(0.5) * R(p.force[0])) / rho, (jy + R(0.5) * R(p.force[1])) / rho,
                    (jz + R(0.5) * R(p.force[2])) / rho};
    R* rho_out = (R*)ib.rho;
    R* us = (R*)ib.u_star;
    rho_out[n] = rho;
#pragma unroll
    for (int a = 0; a < L::D; ++a) us[a * ib.n_nodes + n] = u[a];
    if (s_rho != nullptr) {
        s_rho[n] = rho;
#pragma unroll
        for (int a = 0; a < L::D; ++a) s_us[a * ib.n_nodes + n] = u[a];
    }
}

template <class L, int ST>
__global__ void ibm_moments_kernel(const lbm_grid_t g, const lbm_physics_t p, const lbm_ibm_t ib,
                                   const typename Storage<ST>::T* __restrict__ f, int layout)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < ib.n_nodes) ibm_moments_node<L, ST>(g, p, ib, f, layout, n);
}

// ---------------------------------------------------------------- one launch per step
// Moments and every multi-direct pass of one step in a single block, for
// bodies of up to IBM_FUSED_MAX stencil nodes and markers: phases separated
// by __syncthreads instead of launches. Per pass the marker forces are formed
// once per marker (threads over markers), then spread node-centric (threads
// over nodes) -- the same operations, in the same order, as the per-pass
// kernel, so both paths give the same bits. Buffers written inside the kernel
// are read with plain loads (one block, one SM: its L1 sees its own stores).
// Threads of the block: 512 in 3D, where a marker's 27-node stencil needs
// more registers (no spills at 128 per thread).
template <class L> constexpr int ibm_fused_threads() { return L::D == 2 ? 1024 : 512; }
constexpr int IBM_FUSED_MAX = 4096;

// MODE 1: bodies whose node and marker arrays fit in 48 KB keep a copy of
// them in shared memory (rho, u*, the node force of the previous and the
// current pass, the marker forces of the pass, and each node's velocity
// correction F_n / (2 rho_n) of the previous pass -- formed once per node in
// the node phase, where its divisions run in parallel over the nodes, instead
// of 2 d divisions per stencil entry in every marker's chain: the same
// operands, so the same bits), so the phases read shared memory instead of L2; the global arrays are written as well (the step,
// the body force and the adjoint read them). MODE 2: when the body's tables
// (stencils, weights, areas, the inverse CSR) fit beside them, they are
// copied in too, all with independent loads in one phase, and the passes
// make no global load at all. MODE 0: everything in global memory.
template <class L, int ST>
__host__ __device__ constexpr int64_t ibm_smem_reals(int nn, int nm)
{
    return (int64_t)nn * (1 + 4 * L::D) + (int64_t)L::D * nm;
}
// The tables: real weight[nm S], area[nm], inv_weight[nm S], then int32
// stencil[nm S], inv_start[nn + 1], inv_marker[nm S] (the inverse CSR lists
// every (marker, stencil position) pair once: nm S entries).
template <class L, int ST>
__host__ __device__ constexpr int64_t ibm_table_bytes(int nn, int nm)
{
    constexpr int64_t S = L::D == 2 ? 9 : 27;
    using R = typename Storage<ST>::R;
    return ((int64_t)nm * (2 * S + 1)) * (int64_t)sizeof(R) + ((int64_t)nm * 2 * S + nn + 1) * 4;
}
constexpr int64_t IBM_SMEM_BYTES = 48 * 1024;

template <class L, int ST, int MODE>
__device__ __forceinline__ void ibm_force_block(const lbm_grid_t& g, const lbm_physics_t& p, const lbm_ibm_t& ib,
                                                const typename Storage<ST>::T* __restrict__ f, int layout,
                                                int iterations, typename Storage<ST>::R* force)
{
    using R = typename Storage<ST>::R;
    constexpr int D = L::D;
    constexpr int S = D == 2 ? 9 : 27;
    constexpr bool SMEM = MODE >= 1;
    extern __shared__ __align__(16) unsigned char ibm_smem[];
    const int nn = ib.n_nodes, nm = ib.n_markers;
    R* s_rho = SMEM ? reinterpret_cast<R*>(ibm_smem) : nullptr;
    R* s_us = SMEM ? s_rho + nn : nullptr;
    R* s_f = SMEM ? s_us + D * nn : nullptr;  // two passes: [2][D][nn]
    R* s_mf = SMEM ? s_f + 2 * D * nn : nullptr;
    R* s_corr = SMEM ? s_mf + D * nm : nullptr;  // [D][nn]: F_n / (2 rho_n) of the previous pass
    const int* stencil = ib.stencil;
    const R* wgt = (const R*)ib.weight;
    const R* area = (const R*)ib.area;
    const int* inv_start = ib.inv_start;
    const int* inv_marker = ib.inv_marker;
    const R* invw = (const R*)ib.inv_weight;
    // the thread's first stencil node, loaded ahead of the tables (the moments need it): one round trip fewer
    const int64_t nd0 = (int)threadIdx.x < nn ? ib.node[threadIdx.x] : 0;
    if constexpr (MODE == 2) {
        const int pairs = nm * S;
        R* t_w = s_corr + D * nn;
        R* t_area = t_w + pairs;
        R* t_invw = t_area + nm;
        int* t_st = reinterpret_cast<int*>(t_invw + pairs);
        int* t_is = t_st + pairs;
        int* t_im = t_is + nn + 1;
        const int count = pairs > nn + 1 ? pairs : nn + 1;
        constexpr int U = 4;  // entries per thread per round trip: every load of them first, then the stores
        for (int i0 = threadIdx.x; i0 < count; i0 += U * blockDim.x) {
            int st[U], im[U], is[U];
            R w[U], iw[U], ar[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int i = i0 + u * blockDim.x;
                st[u] = im[u] = is[u] = 0;
                w[u] = iw[u] = ar[u] = R(0);
                if (i < pairs) {
                    st[u] = ib.stencil[i];
                    w[u] = wgt[i];
                    im[u] = ib.inv_marker[i];
                    iw[u] = invw[i];
                }
                if (i <= nn) is[u] = ib.inv_start[i];
                if (i < nm) ar[u] = area[i];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int i = i0 + u * blockDim.x;
                if (i < pairs) {
                    t_st[i] = st[u];
                    t_w[i] = w[u];
                    t_im[i] = im[u];
                    t_invw[i] = iw[u];
                }
                if (i <= nn) t_is[i] = is[u];
                if (i < nm) t_area[i] = ar[u];
            }
        }
        stencil = t_st;
        wgt = t_w;
        area = t_area;
        inv_start = t_is;
        inv_marker = t_im;
        invw = t_invw;
    }
    for (int n = threadIdx.x; n < nn; n += blockDim.x)
        ibm_moments_node<L, ST>(g, p, ib, f, layout, n, s_rho, s_us, n == (int)threadIdx.x ? nd0 : -1);
    __syncthreads();
    const R* rho = SMEM ? s_rho : (const R*)ib.rho;
    const R* us = SMEM ? s_us : (const R*)ib.u_star;
    for (int it = 0; it < iterations; ++it) {
        const R* fin = it == 0 ? nullptr
                               : (SMEM ? s_f + (int64_t)((it - 1) & 1) * D * nn : force + (int64_t)(it - 1) * D * nn);
        R* fout = force + (int64_t)it * D * nn;
        R* s_fout = SMEM ? s_f + (int64_t)(it & 1) * D * nn : nullptr;
        R* mf = (R*)ib.marker_force + (int64_t)it * D * nm;
        const R* mf_read = SMEM ? s_mf : mf;
        for (int l = threadIdx.x; l < nm; l += blockDim.x) {
            const int* st = stencil + (int64_t)l * S;
            const R* wl = wgt + (int64_t)l * S;
            int m[S];
            R w[S];
#pragma unroll
            for (int s = 0; s < S; ++s) {
                m[s] = st[s];
                w[s] = wl[s];
            }
            R rho_l = R(0);
            R U[D];
#pragma unroll
            for (int a = 0; a < D; ++a) U[a] = R(0);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const R rm = rho[m[s]];
                rho_l += w[s] * rm;
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    R u = us[a * nn + m[s]];
                    if (fin != nullptr) u += SMEM ? s_corr[a * nn + m[s]] : fin[a * nn + m[s]] / (R(2) * rm);
                    U[a] += w[s] * u;
                }
            }
#pragma unroll
            for (int a = 0; a < D; ++a) {
                const R Fl = R(2) * rho_l * (R(0) - U[a]) * area[l];
                mf[(int64_t)a * nm + l] = Fl;
                if (SMEM) s_mf[a * nm + l] = Fl;
            }
        }
        __syncthreads();
        for (int n = threadIdx.x; n < nn; n += blockDim.x) {
            double acc[D];
#pragma unroll
            for (int a = 0; a < D; ++a) acc[a] = 0.0;
            for (int q = inv_start[n]; q < inv_start[n + 1]; ++q) {
                const int l = inv_marker[q];
                const R wn = invw[q];
#pragma unroll
                for (int a = 0; a < D; ++a) acc[a] += (double)(wn * mf_read[(int64_t)a * nm + l]);
            }
#pragma unroll
            for (int a = 0; a < D; ++a) {
                const double base = fin != nullptr ? (double)fin[a * nn + n] : 0.0;
                const R v = (R)(base + acc[a]);
                fout[a * nn + n] = v;
                if (SMEM) {
                    s_fout[a * nn + n] = v;
                    s_corr[a * nn + n] = v / (R(2) * rho[n]);  // read by the next pass's markers
                }
            }
        }
        __syncthreads();
    }
}

template <class L, int ST, int MODE>
__global__ void __launch_bounds__(ibm_fused_threads<L>()) ibm_force_fused_kernel(
    const lbm_grid_t g, const lbm_physics_t p, const lbm_ibm_t ib, const typename Storage<ST>::T* __restrict__ f,
    int layout, int iterations, typename Storage<ST>::R* force)
{
    ibm_force_block<L, ST, MODE>(g, p, ib, f, layout, iterations, force);
}

// The immersed-boundary part of a pull step in one block: the body force of
// the step (as ibm_force_fused_kernel), then the update of the special nodes
// of a.sp -- the body's stencil nodes -- with the final pass's node force,
// by the boundary warps' node path (boundary_node: same operations, same
// bits). The last pass ends with a block barrier, after which the node force
// written to global memory is visible to every thread of the block. The step's
// other special nodes and its bulk run in concurrent launches, so no launch of
// the step waits for the force. 512 threads in 2D too: the node update needs
// more than the 64 registers a thread of a 1024-thread block can have.
template <class L> constexpr int ibm_step_threads() { return 512; }

template <class L, int ST, int MODE, int CM>
__global__ void __launch_bounds__(ibm_step_threads<L>()) ibm_step_kernel(const StepArgs a, const lbm_grid_t g,
                                                                          const lbm_physics_t p, const lbm_ibm_t ib,
                                                                          int iterations,
                                                                          typename Storage<ST>::R* force)
{
    ibm_force_block<L, ST, MODE>(g, p, ib, static_cast<const typename Storage<ST>::T*>(a.f_src), LBM_LAYOUT_PULL,
                                 iterations, force);
    for (int64_t s = threadIdx.x; s < a.sp.n_special; s += blockDim.x) boundary_node<L, ST, LBM_PULL, false, CM>(a, s);
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

// The per-pass path of large bodies in two launches, marker-centric then
// node-centric, so that no marker is recomputed: ibm_markers_kernel forms F_l
// of every marker once (the operations of ibm_iteration_kernel, in its order)
// into marker_force[iteration], ibm_spread_kernel adds w_ln F_l over each
// node's CSR list in float64. Same bits as the one-kernel pass.
template <class L, int ST>
__global__ void __launch_bounds__(128) ibm_markers_kernel(const lbm_ibm_t ib, int iteration,
                                                          const typename Storage<ST>::R* __restrict__ fin)
{
    using R = typename Storage<ST>::R;
    constexpr int D = L::D;
    constexpr int S = D == 2 ? 9 : 27;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= ib.n_markers) return;
    const int nn = ib.n_nodes;
    const R* __restrict__ rho = (const R*)ib.rho;
    const R* __restrict__ us = (const R*)ib.u_star;
    const int* st = ib.stencil + (int64_t)l * S;
    const R* wl = (const R*)ib.weight + (int64_t)l * S;
    int m[S];
    R w[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        m[s] = st[s];
        w[s] = wl[s];
    }
    R rho_l = R(0);
    R U[D];
#pragma unroll
    for (int a = 0; a < D; ++a) U[a] = R(0);
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const R rm = rho[m[s]];
        rho_l += w[s] * rm;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            R u = us[a * nn + m[s]];
            if (fin != nullptr) u += fin[a * nn + m[s]] / (R(2) * rm);
            U[a] += w[s] * u;
        }
    }
    R* mf = (R*)ib.marker_force + (int64_t)iteration * D * ib.n_markers;
    const R ar = ((const R*)ib.area)[l];
#pragma unroll
    for (int a = 0; a < D; ++a) mf[(int64_t)a * ib.n_markers + l] = R(2) * rho_l * (R(0) - U[a]) * ar;
}

template <class L, int ST>
__global__ void __launch_bounds__(128) ibm_spread_kernel(const lbm_ibm_t ib, int iteration,
                                                         const typename Storage<ST>::R* __restrict__ fin,
                                                         typename Storage<ST>::R* __restrict__ fout)
{
    using R = typename Storage<ST>::R;
    constexpr int D = L::D;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ib.n_nodes) return;
    const int nn = ib.n_nodes, nm = ib.n_markers;
    const R* __restrict__ mf = (const R*)ib.marker_force + (int64_t)iteration * D * nm;
    const R* __restrict__ invw = (const R*)ib.inv_weight;
    double acc[D];
#pragma unroll
    for (int a = 0; a < D; ++a) acc[a] = 0.0;
    const int q1 = ib.inv_start[n + 1];
    for (int q = ib.inv_start[n]; q < q1; ++q) {
        const int l = ib.inv_marker[q];
        const R wn = invw[q];
#pragma unroll
        for (int a = 0; a < D; ++a) acc[a] += (double)(wn * mf[(int64_t)a * nm + l]);
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

// ---------------------------------------------------------------- adjoint
// Reverse of one pass, node-centric and deterministic like the forward pass:
// node n walks its (marker l, w_ln) list and, per marker, recomputes the
// forward rho_l and U_l of the pass and the adjoint of F_l,
//   Fbar_l = sum_s w_ls adj_in(m(l,s)) - body_scale e_axis,
// from which (F_l = -2 dA_l rho_l U_l, U_l = sum_s w_ls (u*_s + Fp_s / (2 rho_s)))
//   d/dFp_n : -dA_l rho_l w_ln / rho_n
//   d/du*_n : -2 dA_l rho_l w_ln
//   d/drho_n: -2 dA_l w_ln U_l + dA_l rho_l w_ln Fp_n / rho_n^2   (through rho_l and Fp_n / (2 rho_n))
// applied to Fbar_l. Float64 throughout.
template <class L, int ST>
__global__ void ibm_adjoint_iteration_kernel(const lbm_ibm_t ib, const typename Storage<ST>::R* __restrict__ fprev,
                                             const typename Storage<ST>::R* __restrict__ adj_in, int axis,
                                             double body_scale, typename Storage<ST>::R* __restrict__ adj_out,
                                             double* __restrict__ madj)
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
    const double rho_n = (double)rho[n];
    double o[D], ub[D], rb = 0.0;
#pragma unroll
    for (int a = 0; a < D; ++a) o[a] = ub[a] = 0.0;
    for (int p = ib.inv_start[n]; p < ib.inv_start[n + 1]; ++p) {
        const int l = ib.inv_marker[p];
        const int* st = ib.stencil + (int64_t)l * ib.stencil_size;
        const R* wl = wgt + (int64_t)l * ib.stencil_size;
        double rho_l = 0.0, U[D], Fb[D];
#pragma unroll
        for (int a = 0; a < D; ++a) U[a] = Fb[a] = 0.0;
        for (int s = 0; s < ib.stencil_size; ++s) {
            const int m = st[s];
            const double w = (double)wl[s];
            const double rm = (double)rho[m];
            rho_l += w * rm;
#pragma unroll
            for (int a = 0; a < D; ++a) {
                double u = (double)us[a * nn + m];
                if (fprev != nullptr) u += (double)fprev[a * nn + m] / (2.0 * rm);
                U[a] += w * u;
                Fb[a] += w * (double)adj_in[a * nn + m];
            }
        }
        if (axis >= 0 && axis < D) Fb[axis] -= body_scale;
        const double wn = (double)invw[p], dA = (double)area[l];
        const double c = dA * rho_l * wn;
        double UF = 0.0, PF = 0.0;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            o[a] += c * Fb[a];
            ub[a] -= 2.0 * c * Fb[a];
            UF += U[a] * Fb[a];
            if (fprev != nullptr) PF += Fb[a] * (double)fprev[a * nn + n];
        }
        rb += -2.0 * dA * wn * UF + c * PF / (rho_n * rho_n);
    }
    if (adj_out != nullptr) {
#pragma unroll
        for (int a = 0; a < D; ++a) adj_out[a * nn + n] = (R)((double)adj_in[a * nn + n] - o[a] / rho_n);
    }
    madj[n] += rb;
#pragma unroll
    for (int a = 0; a < D; ++a) madj[(int64_t)(1 + a) * nn + n] += ub[a];
}

// The adjoint pass in two launches when the caller gives marker scratch
// (lbm_ibm_t.marker_scratch, (1 + 2 d) doubles per marker): the forward rho_l
// and U_l and the adjoint Fbar_l of each marker once, then the node-centric
// accumulation of ibm_adjoint_iteration_kernel reading them -- the same values
// in the same order, so the same bits, without recomputing each marker for
// every one of its 3^d nodes.
template <class L, int ST>
__global__ void __launch_bounds__(128) ibm_adjoint_markers_kernel(const lbm_ibm_t ib,
                                                                  const typename Storage<ST>::R* __restrict__ fprev,
                                                                  const typename Storage<ST>::R* __restrict__ adj_in,
                                                                  int axis, double body_scale)
{
    using R = typename Storage<ST>::R;
    constexpr int D = L::D;
    constexpr int S = D == 2 ? 9 : 27;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= ib.n_markers) return;
    const int nn = ib.n_nodes, nm = ib.n_markers;
    const R* __restrict__ rho = (const R*)ib.rho;
    const R* __restrict__ us = (const R*)ib.u_star;
    const int* st = ib.stencil + (int64_t)l * S;
    const R* wl = (const R*)ib.weight + (int64_t)l * S;
    int m[S];
    double w[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        m[s] = st[s];
        w[s] = (double)wl[s];
    }
    double rho_l = 0.0, U[D], Fb[D];
#pragma unroll
    for (int a = 0; a < D; ++a) U[a] = Fb[a] = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const double rm = (double)rho[m[s]];
        rho_l += w[s] * rm;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            double u = (double)us[a * nn + m[s]];
            if (fprev != nullptr) u += (double)fprev[a * nn + m[s]] / (2.0 * rm);
            U[a] += w[s] * u;
            Fb[a] += w[s] * (double)adj_in[a * nn + m[s]];
        }
    }
    if (axis >= 0 && axis < D) Fb[axis] -= body_scale;
    double* sc = ib.marker_scratch;
    sc[l] = rho_l;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        sc[(int64_t)(1 + a) * nm + l] = U[a];
        sc[(int64_t)(1 + D + a) * nm + l] = Fb[a];
    }
}

template <class L, int ST>
__global__ void __launch_bounds__(128) ibm_adjoint_nodes_kernel(const lbm_ibm_t ib,
                                                                const typename Storage<ST>::R* __restrict__ fprev,
                                                                const typename Storage<ST>::R* __restrict__ adj_in,
                                                                typename Storage<ST>::R* __restrict__ adj_out,
                                                                double* __restrict__ madj)
{
    using R = typename Storage<ST>::R;
    constexpr int D = L::D;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ib.n_nodes) return;
    const int nn = ib.n_nodes, nm = ib.n_markers;
    const R* __restrict__ area = (const R*)ib.area;
    const R* __restrict__ invw = (const R*)ib.inv_weight;
    const double* __restrict__ sc = ib.marker_scratch;
    const double rho_n = (double)((const R*)ib.rho)[n];
    double fp[D];
#pragma unroll
    for (int a = 0; a < D; ++a) fp[a] = fprev != nullptr ? (double)fprev[a * nn + n] : 0.0;
    double o[D], ub[D], rb = 0.0;
#pragma unroll
    for (int a = 0; a < D; ++a) o[a] = ub[a] = 0.0;
    const int q1 = ib.inv_start[n + 1];
    for (int q = ib.inv_start[n]; q < q1; ++q) {
        const int l = ib.inv_marker[q];
        const double rho_l = sc[l];
        const double wn = (double)invw[q], dA = (double)area[l];
        const double c = dA * rho_l * wn;
        double UF = 0.0, PF = 0.0;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const double U = sc[(int64_t)(1 + a) * nm + l], Fb = sc[(int64_t)(1 + D + a) * nm + l];
            o[a] += c * Fb;
            ub[a] -= 2.0 * c * Fb;
            UF += U * Fb;
            if (fprev != nullptr) PF += Fb * fp[a];
        }
        rb += -2.0 * dA * wn * UF + c * PF / (rho_n * rho_n);
    }
    if (adj_out != nullptr) {
#pragma unroll
        for (int a = 0; a < D; ++a) adj_out[a * nn + n] = (R)((double)adj_in[a * nn + n] - o[a] / rho_n);
    }
    madj[n] += rb;
#pragma unroll
    for (int a = 0; a < D; ++a) madj[(int64_t)(1 + a) * nn + n] += ub[a];
}

// rho = 1 + sum_k s_k, u* = (j + F_uniform / 2) / rho, j = sum_k c_k s_k:
//   d/ds_k = rho_bar - u*_bar . u* / rho + c_k . u*_bar / rho
template <class L, int ST>
__global__ void ibm_adjoint_moments_kernel(const lbm_grid_t g, const lbm_ibm_t ib, double* __restrict__ madj,
                                           typename Storage<ST>::R* __restrict__ mu)
{
    using R = typename Storage<ST>::R;
    constexpr int D = L::D;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ib.n_nodes) return;
    const int nn = ib.n_nodes;
    const R* __restrict__ us = (const R*)ib.u_star;
    const double rho = (double)((const R*)ib.rho)[n];
    double rb = madj[n], jb[3] = {0.0, 0.0, 0.0};
    madj[n] = 0.0;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const double ub = madj[(int64_t)(1 + a) * nn + n];
        madj[(int64_t)(1 + a) * nn + n] = 0.0;
        rb -= ub * (double)us[a * nn + n] / rho;
        jb[a] = ub / rho;
    }
    const int64_t nd = ib.node[n];
#pragma unroll
    for (int k = 0; k < L::Q; ++k) {
        const double v = rb + L::cx(k) * jb[0] + L::cy(k) * jb[1] + L::cz(k) * jb[2];
        mu[(int64_t)k * g.qstride + nd] += (R)v;
    }
}

template <class L, int ST>
int ibm_adjoint_iteration(const lbm_grid_t& g, const lbm_ibm_t& ib, const void* fprev, const void* adj_in, int axis,
                          double body_scale, void* adj_out, double* madj, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    if (ib.n_nodes <= 0) return LBM_OK;
    if (ib.marker_scratch != nullptr) {
        if (ib.n_markers > 0)
            ibm_adjoint_markers_kernel<L, ST><<<blocks_for(ib.n_markers, 128), 128, 0, s>>>(
                ib, (const R*)fprev, (const R*)adj_in, axis, body_scale);
        ibm_adjoint_nodes_kernel<L, ST><<<blocks_for(ib.n_nodes, 128), 128, 0, s>>>(ib, (const R*)fprev,
                                                                                  (const R*)adj_in, (R*)adj_out, madj);
        return launch_status();
    }
    ibm_adjoint_iteration_kernel<L, ST><<<blocks_for(ib.n_nodes, 128), 128, 0, s>>>(
        ib, (const R*)fprev, (const R*)adj_in, axis, body_scale, (R*)adj_out, madj);
    return launch_status();
}

template <class L, int ST>
int ibm_adjoint_moments(const lbm_grid_t& g, const lbm_ibm_t& ib, double* madj, void* mu, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    if (ib.n_nodes <= 0) return LBM_OK;
    ibm_adjoint_moments_kernel<L, ST><<<blocks_for(ib.n_nodes, 128), 128, 0, s>>>(g, ib, madj, (R*)mu);
    return launch_status();
}

template <class L, int ST>
int ibm_moments(const lbm_grid_t& g, const lbm_physics_t& p, const lbm_ibm_t& ib, const void* f, int layout, cudaStream_t s)
{
    if (ib.n_nodes <= 0) return LBM_OK;
    ibm_moments_kernel<L, ST><<<blocks_for(ib.n_nodes, 128), 128, 0, s>>>(g, p, ib, (const typename Storage<ST>::T*)f, layout);
    return launch_status();
}

template <class L, int ST>
int ibm_force(const lbm_grid_t& g, const lbm_physics_t& p, const lbm_ibm_t& ib, const void* f, int layout,
              int iterations, void* force, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    using T = typename Storage<ST>::T;
    if (ib.n_nodes <= 0) return LBM_OK;
    R* out = (R*)force;
    const int64_t smem = ibm_smem_reals<L, ST>(ib.n_nodes, ib.n_markers) * (int64_t)sizeof(R);
    const int64_t with_tables = smem + ibm_table_bytes<L, ST>(ib.n_nodes, ib.n_markers);
    if (with_tables <= IBM_SMEM_BYTES) {
        ibm_force_fused_kernel<L, ST, 2>
            <<<1, ibm_fused_threads<L>(), (size_t)with_tables, s>>>(g, p, ib, (const T*)f, layout, iterations, out);
        return launch_status();
    }
    if (smem <= IBM_SMEM_BYTES) {
        ibm_force_fused_kernel<L, ST, 1>
            <<<1, ibm_fused_threads<L>(), (size_t)smem, s>>>(g, p, ib, (const T*)f, layout, iterations, out);
        return launch_status();
    }
    if (ib.n_nodes <= IBM_FUSED_MAX && ib.n_markers <= IBM_FUSED_MAX) {
        ibm_force_fused_kernel<L, ST, 0>
            <<<1, ibm_fused_threads<L>(), 0, s>>>(g, p, ib, (const T*)f, layout, iterations, out);
        return launch_status();
    }
    ibm_moments_kernel<L, ST><<<blocks_for(ib.n_nodes, 128), 128, 0, s>>>(g, p, ib, (const T*)f, layout);
    const int64_t plane = (int64_t)L::D * ib.n_nodes;
    for (int it = 0; it < iterations; ++it) {
        const R* fin = it == 0 ? nullptr : out + (it - 1) * plane;
        if (ib.n_markers > 0) ibm_markers_kernel<L, ST><<<blocks_for(ib.n_markers, 128), 128, 0, s>>>(ib, it, fin);
        ibm_spread_kernel<L, ST><<<blocks_for(ib.n_nodes, 128), 128, 0, s>>>(ib, it, fin, out + it * plane);
    }
    return launch_status();
}

template <class L, int ST, int CM>
int ibm_step_model(StepArgs a, const lbm_grid_t& g, const lbm_physics_t& p, const lbm_ibm_t& ib, int iterations,
                   void* force, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    R* out = (R*)force;
    a.sp.local_force = out + (int64_t)(iterations - 1) * L::D * ib.n_nodes;  // the final pass
    a.sp.n_local = ib.n_nodes;
    constexpr int threads = ibm_step_threads<L>();
    const int64_t smem = ibm_smem_reals<L, ST>(ib.n_nodes, ib.n_markers) * (int64_t)sizeof(R);
    const int64_t with_tables = smem + ibm_table_bytes<L, ST>(ib.n_nodes, ib.n_markers);
    if (with_tables <= IBM_SMEM_BYTES)
        ibm_step_kernel<L, ST, 2, CM><<<1, threads, (size_t)with_tables, s>>>(a, g, p, ib, iterations, out);
    else if (smem <= IBM_SMEM_BYTES)
        ibm_step_kernel<L, ST, 1, CM><<<1, threads, (size_t)smem, s>>>(a, g, p, ib, iterations, out);
    else if (ib.n_nodes <= IBM_FUSED_MAX && ib.n_markers <= IBM_FUSED_MAX)
        ibm_step_kernel<L, ST, 0, CM><<<1, threads, 0, s>>>(a, g, p, ib, iterations, out);
    else
        return LBM_ERR_UNSUPPORTED;
    return launch_status();
}

template <class L, int ST>
int ibm_step(const StepArgs& a, const lbm_grid_t& g, const lbm_physics_t& p, const lbm_ibm_t& ib, int iterations,
             void* force, cudaStream_t s)
{
    if (a.collision == LBM_COLLIDE_REGULARIZED)
        return ibm_step_model<L, ST, LBM_COLLIDE_REGULARIZED>(a, g, p, ib, iterations, force, s);
    if (a.collision == LBM_COLLIDE_CUMULANT) {
        if constexpr (L::D == 2) return ibm_step_model<L, ST, LBM_COLLIDE_CUMULANT>(a, g, p, ib, iterations, force, s);
        return LBM_ERR_UNSUPPORTED;
    }
    return ibm_step_model<L, ST, LBM_COLLIDE_TRT>(a, g, p, ib, iterations, force, s);
}

template <class L, int ST>
int ibm_iteration(const lbm_grid_t& g, const lbm_ibm_t& ib, int iteration, const void* fin, void* fout, cudaStream_t s)
{
    using R = typename Storage<ST>::R;
    if (ib.n_nodes <= 0) return LBM_OK;
    if (ib.n_markers > 0)
        ibm_markers_kernel<L, ST><<<blocks_for(ib.n_markers, 128), 128, 0, s>>>(ib, iteration, (const R*)fin);
    ibm_spread_kernel<L, ST><<<blocks_for(ib.n_nodes, 128), 128, 0, s>>>(ib, iteration, (const R*)fin, (R*)fout);
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
    if (!grid_valid(g) || !ib || ib->n_nodes < 0 || ib->n_markers < 0) return false;
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

extern "C" int lbm_ibm_force(const lbm_grid_t* g, const lbm_physics_t* p, const lbm_ibm_t* ib, const void* f,
                             int32_t layout, int32_t iterations, void* force, lbm_stream_t stream)
{
    if (!ibm_ok(g, ib) || !p || !f || !force || iterations < 1) return LBM_ERR_INVALID;
    if (layout < LBM_LAYOUT_PULL || layout > LBM_LAYOUT_AA_EVEN) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, ibm_force, *g, *p, *ib, f, layout, iterations, force, (cudaStream_t)stream);
}

extern "C" int lbm_step_pull_ibm(const lbm_grid_t* g, const lbm_physics_t* p, const lbm_special_t* sp,
                                 const lbm_ibm_t* ib, int32_t iterations, const uint8_t* kind, const void* f_src,
                                 void* f_dst, void* force, lbm_stream_t stream)
{
    if (!grid_valid(g) || !ibm_ok(g, ib) || !p || !sp || !kind || !f_src || !f_dst || f_src == f_dst || !force ||
        iterations < 1 || !special_valid(sp, false))
        return LBM_ERR_INVALID;
    if (ib->n_nodes <= 0 || (sp->n_special > 0 && !sp->force_slot)) return LBM_ERR_INVALID;
    StepArgs a;
    int tx = 0, ty = 0, mode = 0;
    const int st = make_args(a, g, p, sp, nullptr, kind, f_src, f_dst, tx, ty, mode);
    if (st != LBM_OK) return st;
    a.parity = (uintptr_t)f_src > (uintptr_t)f_dst ? 1 : 0;
    LBM_DISPATCH(g->lattice, g->storage, ibm_step, a, *g, *p, *ib, iterations, force, (cudaStream_t)stream);
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

extern "C" int lbm_ibm_adjoint_iteration(const lbm_grid_t* g, const lbm_ibm_t* ib, const void* force_prev,
                                         const void* adj_in, int32_t axis, double body_scale, void* adj_out,
                                         double* moment_adj, lbm_stream_t stream)
{
    if (!ibm_ok(g, ib) || !adj_in || !moment_adj || adj_in == adj_out) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, ibm_adjoint_iteration, *g, *ib, force_prev, adj_in, axis, body_scale, adj_out,
                 moment_adj, (cudaStream_t)stream);
}

extern "C" int lbm_ibm_adjoint_moments(const lbm_grid_t* g, const lbm_ibm_t* ib, double* moment_adj, void* mu,
                                       lbm_stream_t stream)
{
    if (!ibm_ok(g, ib) || !moment_adj || !mu) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, ibm_adjoint_moments, *g, *ib, moment_adj, mu, (cudaStream_t)stream);
}
