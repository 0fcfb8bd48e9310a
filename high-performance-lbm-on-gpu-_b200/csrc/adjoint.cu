// Reverse mode of the two-lattice step: one fused kernel per backward step.
//
// Forward step at a fluid node x (pull layout, reference src/lbm/solver.py:257-274):
//   s_k(x) = f_t[k](x - c_k), or f_t[opp k](x) + Ladd term if x - c_k is solid,
//            or a link rule  const + sum coeff * f_t[slot];
//   f_{t+1}(x) = C(s(x), F(x))        (TRT + Guo, csrc/lbm_common.cuh)
// Backward: with lambda_{t+1} the adjoint of f_{t+1} and mu_t = J_C^T lambda_{t+1}
// (the adjoint of s_t), the transposed streaming gives
//   lambda_t[k](y) = mu_t[k](y + c_k)                 if y + c_k is fluid,
//                  = mu_t[opp k](y)                    if it is solid (bounce-back)
//                    unless the link (y, opp k) carries a rule,
//                  + sum over rule terms reading f_t[k](y) of coeff * mu_t[j](x)
//                  + dL/df_t[k](y)                     (force-probe loss).
// The kernel for step t fuses the transposed streaming of mu_{t+1} (giving
// lambda_{t+1} at x) with the transposed collision at x (giving mu_t), so
// lambda is never stored: it reads f_t and mu_{t+1} and writes mu_t.
//
// Transposed collision, in closed form. With w-weighted moments of lambda
//   L0 = sum w_i l_i,  L1 = sum w_i c_i l_i,  L2 = sum w_i c_i c_i^T l_i,
// and the factored update f*_i = a s_i + b s_opp(i) + w_i h(c_i.u, c_i.F)
// (lbm_common.cuh), H = sum l_i w_i h_i = A L0 + B u.L2.u + C u.L2.F + D u.L1 + G F.L1:
//   Hu   = dH/du       = L0 (-3 w+ rho u - 3 (1 - w+/2) F) + 2 B L2 u + C L2 F + D L1
//   Hrho = dH/ddrho|u  = L0 w+ (1 - 1.5 u.u) + 4.5 w+ u.L2.u + 3 w- u.L1
//   HF   = dH/dF|u     = -3 (1 - w+/2) u L0 + C L2 u + G L1
//   mu_k = a l_k + b l_opp(k) + Hrho + (c_k - u).Hu / rho       (du/ds_k = (c_k - u)/rho)
//   dL/dF = HF + Hu / (2 rho)                                    (du/dF = 1/(2 rho))
#include "dispatch.cuh"
#include "step_kernels.cuh"

namespace lbm {

struct AdjArgs {
    StepArgs a;  // f_src = f_t
    lbm_adjoint_t adj;
    const void* mu_next;
    void* mu_out;
    double loss_scale;
};

template <class L, class R>
__device__ __forceinline__ void collide_vjp(const R (&s)[L::Q], R (&lam)[L::Q], R wp, R wm, const R (&F)[3], R (&g)[3])
{
    constexpr int Q = L::Q;
    R drho = s[0], jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        drho += s[i];
        if (L::cx(i) > 0) jx += s[i];
        if (L::cx(i) < 0) jx -= s[i];
        if (L::cy(i) > 0) jy += s[i];
        if (L::cy(i) < 0) jy -= s[i];
        if (L::cz(i) > 0) jz += s[i];
        if (L::cz(i) < 0) jz -= s[i];
    }
    const R rho = R(1) + drho;
    const R inv = R(1) / rho;
    const R u[3] = {(jx + R(0.5) * F[0]) * inv, (jy + R(0.5) * F[1]) * inv, L::D == 3 ? (jz + R(0.5) * F[2]) * inv : R(0)};
    const R usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const R ap = R(1) - R(0.5) * wp, am = R(1) - R(0.5) * wm;
    const R B = R(4.5) * wp * rho, C = R(9) * ap, Dm = R(3) * wm * rho, G = R(3) * am;
    const R ca = R(1) - R(0.5) * (wp + wm), cb = R(0.5) * (wm - wp);

    R L0 = R(0), L1[3] = {R(0), R(0), R(0)}, L2[3][3] = {{R(0), R(0), R(0)}, {R(0), R(0), R(0)}, {R(0), R(0), R(0)}};
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const R wl = R(L::w(i)) * lam[i];
        const int c[3] = {L::cx(i), L::cy(i), L::cz(i)};
        L0 += wl;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (c[a] == 0) continue;
            L1[a] += c[a] > 0 ? wl : -wl;
#pragma unroll
            for (int b = a; b < 3; ++b)
                if (c[b] != 0) L2[a][b] += (c[a] * c[b] > 0) ? wl : -wl;
        }
    }
    L2[1][0] = L2[0][1];
    L2[2][0] = L2[0][2];
    L2[2][1] = L2[1][2];
    R L2u[3], L2F[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        L2u[a] = L2[a][0] * u[0] + L2[a][1] * u[1] + L2[a][2] * u[2];
        L2F[a] = L2[a][0] * F[0] + L2[a][1] * F[1] + L2[a][2] * F[2];
    }
    const R uL2u = u[0] * L2u[0] + u[1] * L2u[1] + u[2] * L2u[2];
    const R uL1 = u[0] * L1[0] + u[1] * L1[1] + u[2] * L1[2];
    R Hu[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
        Hu[a] = L0 * (R(-3) * wp * rho * u[a] - R(3) * ap * F[a]) + R(2) * B * L2u[a] + C * L2F[a] + Dm * L1[a];
    const R Hrho = L0 * wp * (R(1) - R(1.5) * usq) + R(4.5) * wp * uL2u + R(3) * wm * uL1;
    const R V[3] = {Hu[0] * inv, Hu[1] * inv, Hu[2] * inv};
    const R P = Hrho - (u[0] * V[0] + u[1] * V[1] + u[2] * V[2]);
#pragma unroll
    for (int a = 0; a < 3; ++a) g[a] = R(-3) * ap * u[a] * L0 + C * L2u[a] + G * L1[a] + R(0.5) * V[a];
    lam[0] = (ca + cb) * lam[0] + P;
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        const int o = L::opp(i);
        if (o < i) continue;
        const R cv = R(L::cx(i)) * V[0] + R(L::cy(i)) * V[1] + R(L::cz(i)) * V[2];
        const R li = lam[i], lo = lam[o];
        lam[i] = ca * li + cb * lo + P + cv;
        lam[o] = ca * lo + cb * li + P - cv;
    }
}

template <class L, int ST>
struct AdjointKernel {
    using S = Storage<ST>;
    using T = typename S::T;
    using R = typename S::R;
    static constexpr int Q = L::Q;

    __device__ static __forceinline__ void force_at(const StepArgs& a, int64_t nd, R (&F)[3])
    {
        F[0] = R(a.fx);
        F[1] = R(a.fy);
        F[2] = R(a.fz);
        if (a.force_field != nullptr) {
            const R* ff = static_cast<const R*>(a.force_field);
            F[0] += ff[nd];
            F[1] += ff[a.qstride + nd];
            if (L::D == 3) F[2] += ff[2 * a.qstride + nd];
        }
    }

    // s_idx >= 0: node of the special list; its force slot (immersed-boundary
    // stencil nodes) adds the recomputed node force, and dL/dF there goes to
    // local_force_grad for the immersed-boundary adjoint.
    __device__ static __forceinline__ void finish(const AdjArgs& A, int64_t nd, const R (&s)[Q], R (&lam)[Q],
                                                  int64_t s_idx = -1)
    {
        const StepArgs& a = A.a;
        R F[3], g[3];
        force_at(a, nd, F);
        const int fs = s_idx >= 0 && a.sp.force_slot != nullptr ? a.sp.force_slot[s_idx] : -1;
        if (fs >= 0) {
            const R* lf = static_cast<const R*>(a.sp.local_force);
            const int64_t n = a.sp.n_local;
#pragma unroll
            for (int c = 0; c < L::D; ++c) F[c] += lf[c * n + fs];
        }
        collide_vjp<L, R>(s, lam, R(a.wp), R(a.wm), F, g);
        R* mu = static_cast<R*>(A.mu_out) + nd;
#pragma unroll
        for (int i = 0; i < Q; ++i) mu[i * a.qstride] = lam[i];
        if (A.adj.force_grad != nullptr) {
            R* fg = static_cast<R*>(A.adj.force_grad) + nd;
#pragma unroll
            for (int c = 0; c < L::D; ++c) fg[c * a.qstride] += g[c];
        }
        if (fs >= 0 && A.adj.local_force_grad != nullptr) {
            R* lg = static_cast<R*>(A.adj.local_force_grad);
#pragma unroll
            for (int c = 0; c < L::D; ++c) lg[c * (int64_t)a.sp.n_local + fs] = g[c];
        }
    }

    // Interior node: lambda_k = mu_next[k](x + c_k), s_k = f_t[k](x - c_k).
    __device__ static __forceinline__ void interior(const AdjArgs& A, int64_t nd)
    {
        const StepArgs& a = A.a;
        const int64_t qs = a.qstride, py = a.pitch, pz = (int64_t)a.pitch * a.ny;
        R s[Q], lam[Q];
        const T* fs = static_cast<const T*>(a.f_src) + nd;
        const R* mn = static_cast<const R*>(A.mu_next);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int64_t shift = L::cx(i) + L::cy(i) * py + L::cz(i) * pz;
            s[i] = S::load_nc(fs + (i * qs - shift));
            lam[i] = mn != nullptr ? __ldg(mn + nd + (i * qs + shift)) : R(0);
        }
        finish(A, nd, s, lam);
    }

    // Rule r and its U-derivative from one pass over the term loads:
    // v = const + sum coeff f (as rule_value), d = dconst + sum dcoeff f in
    // float64. Loads issued sixteen terms at a time (last batch predicated).
    __device__ static __forceinline__ void rule_value_du(const AdjArgs& A, int r, R& v, double& d)
    {
        constexpr int B = 16;
        const StepArgs& a = A.a;
        const lbm_special_t& sp = a.sp;
        const R* __restrict__ coeff = static_cast<const R*>(sp.term_coeff);
        const R* __restrict__ dcoeff = static_cast<const R*>(A.adj.term_dcoeff);
        const T* __restrict__ f = static_cast<const T*>(a.f_src);
        v = static_cast<const R*>(sp.rule_const)[r];
        d = (double)static_cast<const R*>(A.adj.rule_dconst)[r];
        const int t1 = sp.term_start[r + 1];
        for (int t = sp.term_start[r]; t < t1; t += B) {
            int64_t slot[B];
            R c[B], dc[B], val[B];
#pragma unroll
            for (int k = 0; k < B; ++k) {
                const bool in = t + k < t1;
                slot[k] = in ? (int64_t)sp.term_dir[t + k] * a.qstride + sp.term_node[t + k] : 0;
                c[k] = in ? coeff[t + k] : R(0);
                dc[k] = in ? dcoeff[t + k] : R(0);
            }
#pragma unroll
            for (int k = 0; k < B; ++k) val[k] = S::load(f + slot[k]);
#pragma unroll
            for (int k = 0; k < B; ++k)
                if (t + k < t1) {
                    v = v_fma(c[k], val[k], v);
                    d += (double)dc[k] * (double)val[k];
                }
        }
    }

    // The node's rules in the dense form: distinct term values loaded once,
    // then per rule its value (coefficient row) and, with a U-derivative, the
    // derivative row in float64 -- as rule_value_du, in two memory round trips
    // for all the node's rules.
    __device__ static __forceinline__ void dense_rules_du(const AdjArgs& A, int64_t s_idx, uint32_t rmask, int rfirst,
                                                          bool with_du, R (&s)[Q], double (&dv)[Q])
    {
        constexpr int UM = LBM_DENSE_TERMS;
        const StepArgs& a = A.a;
        const lbm_special_t& sp = a.sp;
        const int u0 = sp.ut_start[s_idx];
        const int n = sp.ut_start[s_idx + 1] - u0;
        const T* __restrict__ f = static_cast<const T*>(a.f_src);
        int64_t slot[UM];
        R v[UM];
#pragma unroll
        for (int u = 0; u < UM; ++u) slot[u] = u < n ? sp.ut_slot[u0 + u] : -1;
#pragma unroll
        for (int u = 0; u < UM; ++u) v[u] = slot[u] >= 0 ? S::load(f + slot[u]) : R(0);
        // the rows of the node's rules are consecutive, (n + 3) & ~3 apart
        const int64_t row0 = sp.rule_row[rfirst];
        const R* __restrict__ dense = static_cast<const R*>(sp.rule_dense) + row0;
        const R* __restrict__ ddense = static_cast<const R*>(A.adj.rule_ddense) + row0;
        const R* __restrict__ rconst = static_cast<const R*>(sp.rule_const);
        const R* __restrict__ dconst = static_cast<const R*>(A.adj.rule_dconst);
        const int n4 = (n + 3) & ~3;
        uint32_t m = rmask;
        int r = rfirst;
        int row = 0;
        while (m) {
            const int i = __ffs(m) - 1;
            m &= m - 1u;
            R acc = rconst[r];
            double d = with_du ? (double)dconst[r] : 0.0;
#pragma unroll
            for (int u = 0; u < UM; u += 4) {
                if (u < n) {
                    R c[4];
                    load4(dense + row + u, c);
#pragma unroll
                    for (int k = 0; k < 4; ++k) acc = v_fma(c[k], v[u + k], acc);
                    if (with_du) {
                        load4(ddense + row + u, c);
#pragma unroll
                        for (int k = 0; k < 4; ++k) d += (double)c[k] * (double)v[u + k];
                    }
                }
            }
            ++r;
            row += n4;
#pragma unroll
            for (int j = 0; j < Q; ++j)
                if (j == i) {
                    s[j] = acc;
                    dv[j] = d;
                }
        }
    }

    // Any fluid node that is not interior: bounce-back and wrap; for nodes of
    // the adjoint list (s_idx >= 0) also rules, rule-term and loss gathers.
    // acc: this thread's column of a shared [Q][BOUNDARY_THREADS] array
    // (boundary kernel; nullptr in the bulk kernel, which has no gathers).
    __device__ static __forceinline__ void general(const AdjArgs& A, int64_t nd, int64_t s_idx, R* acc)
    {
        const StepArgs& a = A.a;
        const lbm_special_t& sp = a.sp;
        const int64_t row = nd / a.pitch;
        const int x = (int)(nd - row * a.pitch), y = (int)(row % a.ny), z = (int)(row / a.ny);
        const int64_t qs = a.qstride;
        const uint32_t bb = a.nbr[nd];
        // Rule-term and loss gathers into lambda, first (nothing else is live
        // yet, so a batch can be wide): accumulated per direction in shared
        // memory (a runtime direction index; in registers it would be a select
        // over all Q directions per entry), added to lambda before the VJP.
        // Entries thirty-two at a time: metadata, then the mu values.
        if (s_idx >= 0) {
            constexpr int BT = BOUNDARY_THREADS;
#pragma unroll
            for (int j = 0; j < Q; ++j) acc[j * BT] = R(0);
            constexpr int B = 32;
            const R* gc = static_cast<const R*>(A.adj.gather_coeff);
            const R scale = R(A.loss_scale);
            const R* mg = static_cast<const R*>(A.mu_next);
            const int e1 = A.adj.gather_start[s_idx + 1];
            for (int e0 = A.adj.gather_start[s_idx]; e0 < e1; e0 += B) {
                int64_t slot[B];
                int dir[B];
                R c[B], val[B];
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const bool in = e0 + k < e1;
                    slot[k] = in ? A.adj.gather_slot[e0 + k] : -1;
                    dir[k] = in ? A.adj.gather_dir[e0 + k] : 0;
                    c[k] = in ? gc[e0 + k] : R(0);
                }
#pragma unroll
                for (int k = 0; k < B; ++k) val[k] = (slot[k] >= 0 && mg != nullptr) ? mg[slot[k]] : R(0);
#pragma unroll
                for (int k = 0; k < B; ++k)
                    if (e0 + k < e1) acc[dir[k] * BT] += slot[k] >= 0 ? c[k] * val[k] : c[k] * scale;
            }
        }

        const uint32_t rmask = s_idx >= 0 ? sp.rule_mask[s_idx] : 0u;
        const int rfirst = s_idx >= 0 ? sp.rule_first[s_idx] : 0;
        const int xm = wrap(x - 1, a.nx), xp = wrap(x + 1, a.nx);
        const int ym = wrap(y - 1, a.ny), yp = wrap(y + 1, a.ny);
        const int zm = L::D == 3 ? wrap(z - 1, a.nz) : 0, zp = L::D == 3 ? wrap(z + 1, a.nz) : 0;
        const T* f = static_cast<const T*>(a.f_src);
        const R* mn = static_cast<const R*>(A.mu_next);
        const R* wall = static_cast<const R*>(a.wall_u);
        R s[Q], lam[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            // forward: streamed s_i from x - c_i
            const int sx = L::cx(i) > 0 ? xm : (L::cx(i) < 0 ? xp : x);
            const int sy = L::cy(i) > 0 ? ym : (L::cy(i) < 0 ? yp : y);
            const int sz = L::cz(i) > 0 ? zm : (L::cz(i) < 0 ? zp : z);
            const int64_t src = ((int64_t)sz * a.ny + sy) * a.pitch + sx;
            if (i != 0 && ((bb >> i) & 1u))
                s[i] = v_add(S::load(f + L::opp(i) * qs + nd), wall_term<L, R>(i, wall, src, qs));
            else
                s[i] = S::load(f + i * qs + src);
            // backward: lambda_i from x + c_i
            lam[i] = R(0);
            if (mn != nullptr) {
                const int dx = L::cx(i) > 0 ? xp : (L::cx(i) < 0 ? xm : x);
                const int dy = L::cy(i) > 0 ? yp : (L::cy(i) < 0 ? ym : y);
                const int dz = L::cz(i) > 0 ? zp : (L::cz(i) < 0 ? zm : z);
                const int64_t dst = ((int64_t)dz * a.ny + dy) * a.pitch + dx;
                if (i == 0 || !((bb >> L::opp(i)) & 1u))
                    lam[i] = mn[i * qs + dst];
                else if (!((rmask >> L::opp(i)) & 1u))
                    lam[i] = mn[L::opp(i) * qs + nd];
            }
        }
        // rules replace bounce-back values in the forward gather; with a
        // U-derivative the same term loads also give d(rule)/dU (dv)
        const bool with_du = A.adj.rule_du != nullptr && A.adj.rule_dconst != nullptr;
        double dv[Q];
#pragma unroll
        for (int j = 0; j < Q; ++j) dv[j] = 0.0;
        if (rmask && sp.ut_start != nullptr && (!with_du || A.adj.rule_ddense != nullptr)) {
            dense_rules_du(A, s_idx, rmask, rfirst, with_du, s, dv);
        } else {
            uint32_t m = rmask;
            int r = rfirst;
            while (m) {
                const int i = __ffs(m) - 1;
                m &= m - 1u;
                R v;
                double d = 0.0;
                if (with_du)
                    rule_value_du(A, r, v, d);
                else
                    v = StepKernel<L, ST, LBM_PULL>::rule_value(a, r);
                ++r;
#pragma unroll
                for (int j = 0; j < Q; ++j)
                    if (j == i) {
                        s[j] = v;
                        dv[j] = d;
                    }
            }
        }
        if (s_idx >= 0) {
#pragma unroll
            for (int j = 0; j < Q; ++j) lam[j] += acc[j * BOUNDARY_THREADS];
        }
        finish(A, nd, s, lam, s_idx);  // lam now holds mu_t at x
        // d rule value / dU, weighted by mu of the ruled direction: the
        // node's accumulators (consecutive rules) loaded at once, then stored
        if (with_du && rmask) {
            double* __restrict__ du = A.adj.rule_du + rfirst;
            double old[Q];
            int k = 0;
#pragma unroll
            for (int i = 0; i < Q; ++i)
                if ((rmask >> i) & 1u) old[i] = du[k++];
            k = 0;
#pragma unroll
            for (int i = 0; i < Q; ++i)
                if ((rmask >> i) & 1u) du[k++] = __fma_rn((double)lam[i], dv[i], old[i]);
        }
    }
};

// 4 resident blocks of 256 (64 registers) for 4-byte reals, where that costs
// a few bytes of spill; float64 would spill ~900 bytes per thread there.
template <int ST>
constexpr int adjoint_bulk_min_blocks()
{
    return sizeof(typename Storage<ST>::R) == 4 ? 4 : 1;
}

template <class L, int ST>
__global__ void __launch_bounds__(256, adjoint_bulk_min_blocks<ST>()) lbm_adjoint_bulk_kernel(const AdjArgs A)
{
    const StepArgs& a = A.a;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.nx || y >= a.ny) return;
    const int64_t nd = ((int64_t)blockIdx.z * a.ny + y) * a.pitch + x;
    const uint8_t k = a.kind[nd];
    if (k == KIND_FLUID)
        AdjointKernel<L, ST>::interior(A, nd);
    else if (!(k & (KIND_SOLID | KIND_SPECIAL)))
        AdjointKernel<L, ST>::general(A, nd, -1, nullptr);
}

template <class L, int ST>
__global__ void __launch_bounds__(256, 1) lbm_adjoint_boundary_kernel(const AdjArgs A)
{
    using R = typename Storage<ST>::R;
    __shared__ R acc[L::Q * BOUNDARY_THREADS];
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s < A.a.sp.n_special) AdjointKernel<L, ST>::general(A, A.a.sp.node[s], s, acc + threadIdx.x);
}

template <class L, int ST>
int adjoint_step(const AdjArgs& A, int mode, int tile_x, int tile_y, cudaStream_t s)
{
    const StepArgs& a = A.a;
    if (mode != LBM_LAUNCH_BOUNDARY) {
        if (a.nz > 65535) return LBM_ERR_INVALID;
        const dim3 grid((a.nx + tile_x - 1) / tile_x, (a.ny + tile_y - 1) / tile_y, a.nz);
        lbm_adjoint_bulk_kernel<L, ST><<<grid, dim3(tile_x, tile_y), 0, s>>>(A);
    }
    if (mode != LBM_LAUNCH_BULK && a.sp.n_special > 0)
        lbm_adjoint_boundary_kernel<L, ST>
            <<<(unsigned)((a.sp.n_special + BOUNDARY_THREADS - 1) / BOUNDARY_THREADS), BOUNDARY_THREADS, 0, s>>>(A);
    return launch_status();
}

// lambda_0 from mu_0, then the derivative of the initial equilibrium
// (velocity u0 + F/(2 rho0)) w.r.t. the per-node force.
template <class L, int ST>
__global__ void lbm_adjoint_initial_kernel(const AdjArgs A, const double* __restrict__ rho0, const double* __restrict__ u0)
{
    using R = typename Storage<ST>::R;
    constexpr int Q = L::Q;
    const StepArgs& a = A.a;
    const int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (nd >= a.qstride || A.adj.force_grad == nullptr) return;
    const int64_t row = nd / a.pitch;
    const int x = (int)(nd - row * a.pitch), y = (int)(row % a.ny), z = (int)(row / a.ny);
    if (x >= a.nx || (a.kind[nd] & KIND_SOLID)) return;
    const int64_t qs = a.qstride;
    const R* mn = static_cast<const R*>(A.mu_next);
    // lambda_0 at this node: same transposed streaming as the step
    R lam[Q];
    const bool special = (a.kind[nd] & KIND_SPECIAL) != 0;
    int64_t sidx = -1;
    if (special) {
        int64_t lo = 0, hi = a.sp.n_special - 1;  // the list is sorted
        while (lo <= hi) {
            const int64_t mid = (lo + hi) / 2;
            const int64_t v = a.sp.node[mid];
            if (v == nd) { sidx = mid; break; }
            if (v < nd) lo = mid + 1; else hi = mid - 1;
        }
    }
    const uint32_t rmask = sidx >= 0 ? a.sp.rule_mask[sidx] : 0u;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int dx = wrap(x + L::cx(i), a.nx), dy = wrap(y + L::cy(i), a.ny);
        const int dz = L::D == 3 ? wrap(z + L::cz(i), a.nz) : 0;
        const int64_t dst = ((int64_t)dz * a.ny + dy) * a.pitch + dx;
        if (i == 0 || !(a.kind[dst] & KIND_SOLID))
            lam[i] = mn[i * qs + dst];
        else
            lam[i] = ((rmask >> L::opp(i)) & 1u) ? R(0) : mn[L::opp(i) * qs + nd];
    }
    if (sidx >= 0) {
        const R* gc = static_cast<const R*>(A.adj.gather_coeff);
        for (int e = A.adj.gather_start[sidx]; e < A.adj.gather_start[sidx + 1]; ++e) {
            const int64_t slot = A.adj.gather_slot[e];
            const R v = slot >= 0 ? gc[e] * mn[slot] : gc[e] * R(A.loss_scale);
            const int k = A.adj.gather_dir[e];
#pragma unroll
            for (int j = 0; j < Q; ++j)
                if (j == k) lam[j] += v;
        }
    }
    // f_0 = feq(rho0, u'), u' = u0 + F/(2 rho0); d feq_k / d u'_a = w_k rho (3 c_ka + 9 (c_k.u') c_ka - 3 u'_a)
    R F[3];
    AdjointKernel<L, ST>::force_at(a, nd, F);
    const double r0 = rho0[nd];
    R up[3] = {R(0), R(0), R(0)};
    for (int c = 0; c < L::D; ++c) up[c] = (R)(u0[c * qs + nd] + 0.5 * (double)F[c] / r0);
    const R rho = R(1) + (R)(r0 - 1.0);
    R grad[3] = {R(0), R(0), R(0)};
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const R cu = R(L::cx(k)) * up[0] + R(L::cy(k)) * up[1] + R(L::cz(k)) * up[2];
        const int c[3] = {L::cx(k), L::cy(k), L::cz(k)};
        const R wl = R(L::w(k)) * rho * lam[k];
#pragma unroll
        for (int d = 0; d < 3; ++d) grad[d] += wl * (R(3) * R(c[d]) + R(9) * cu * R(c[d]) - R(3) * up[d]);
    }
    R* fg = static_cast<R*>(A.adj.force_grad) + nd;
    for (int c = 0; c < L::D; ++c) fg[c * qs] += grad[c] * (R(0.5) / (R)r0);
}

template <class L, int ST>
int adjoint_initial(const AdjArgs& A, const double* rho0, const double* u0, cudaStream_t s)
{
    lbm_adjoint_initial_kernel<L, ST><<<blocks_for(A.a.qstride, 256), 256, 0, s>>>(A, rho0, u0);
    return launch_status();
}

}  // namespace lbm

using namespace lbm;

static bool make_adj(AdjArgs& A, const lbm_grid_t* g, const lbm_physics_t* p, const lbm_special_t* sp,
                     const lbm_adjoint_t* adj, const uint8_t* kind, const void* f_t, const void* mu_next, void* mu_out,
                     double loss_scale)
{
    if (!grid_valid(g) || !p || !adj || !kind) return false;
    if (p->collision != LBM_COLLIDE_TRT) return false;  // the transposed collision is TRT/BGK's
    StepArgs& a = A.a;
    a.nx = g->nx;
    a.ny = g->ny;
    a.nz = g->nz;
    a.pitch = g->pitch;
    a.qstride = g->qstride;
    a.wp = p->omega_plus;
    a.wm = p->omega_minus;
    a.fx = p->force[0];
    a.fy = p->force[1];
    a.fz = g->lattice == LBM_D3Q19 ? p->force[2] : 0.0;
    a.kind = kind;
    a.f_src = f_t;
    a.f_dst = nullptr;
    a.wall_u = p->wall_u;
    a.force_field = p->force_field;
    a.nbr = p->solid_nbr;
    if (!a.nbr) return false;
    if (sp)
        a.sp = *sp;
    else
        memset(&a.sp, 0, sizeof(a.sp));
    if (a.sp.n_special > 0 && (!adj->gather_start || !a.sp.node || !a.sp.rule_mask || !a.sp.rule_first)) return false;
    if (a.sp.n_local > 0 && a.sp.n_special > 0 && (!a.sp.force_slot || !a.sp.local_force)) return false;
    A.adj = *adj;
    A.mu_next = mu_next;
    A.mu_out = mu_out;
    A.loss_scale = loss_scale;
    return true;
}

extern "C" int lbm_adjoint_step(const lbm_grid_t* g, const lbm_physics_t* p, const lbm_special_t* sp,
                                const lbm_adjoint_t* adj, const lbm_launch_t* launch, const uint8_t* kind,
                                const void* f_t, const void* mu_next, void* mu_out, double loss_scale,
                                lbm_stream_t stream)
{
    AdjArgs A;
    if (!f_t || !mu_out || mu_out == mu_next || !make_adj(A, g, p, sp, adj, kind, f_t, mu_next, mu_out, loss_scale))
        return LBM_ERR_INVALID;
    const int tx = launch ? launch->tile_x : 32, ty = launch ? launch->tile_y : 4;
    const int mode = launch ? launch->mode : LBM_LAUNCH_FUSED;
    if (tx <= 0 || ty <= 0 || tx % 32 || tx * ty > 256) return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, adjoint_step, A, mode, tx, ty, (cudaStream_t)stream);
}

extern "C" int lbm_adjoint_initial(const lbm_grid_t* g, const lbm_physics_t* p, const lbm_special_t* sp,
                                   const lbm_adjoint_t* adj, const uint8_t* kind, const void* mu0, const double* rho0,
                                   const double* u0, double loss_scale, lbm_stream_t stream)
{
    AdjArgs A;
    if (!mu0 || !rho0 || !u0 || !make_adj(A, g, p, sp, adj, kind, nullptr, mu0, nullptr, loss_scale))
        return LBM_ERR_INVALID;
    LBM_DISPATCH(g->lattice, g->storage, adjoint_initial, A, rho0, u0, (cudaStream_t)stream);
}
