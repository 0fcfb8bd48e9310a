// The fused LBM time step: two-lattice pull and in-place AA, D2Q9/D3Q19,
// float32/float64/float16/bfloat16 storage.
//
// One launch updates every fluid node once:
//   * bulk blocks: a (tile_x x tile_y) tile of one z plane, one node per
//     thread. Warps of interior nodes (kind 0) stream with fixed,
//     warp-uniform offsets and no branch; a warp with a node next to a wall
//     or on a periodic face takes the general path on all its lanes, driven
//     by the precomputed solid-neighbour mask (no neighbour kind is loaded,
//     so all loads stay independent).
//   * boundary warps: one thread per SPECIAL node of the compact list --
//     carrying link rules, an immersed-boundary force or AA rule-term
//     exports. Rules are evaluated in registers while the node is updated,
//     so they need no pre-pass launch and no scatter.
//   The boundary warps run in the same launch (FUSED) or as a second kernel
//   that may overlap the bulk (BULK + BOUNDARY); see lbm_launch_t.
//
// Race freedom.
//   Pull: f_src is never written; rules read it directly.
//   AA (reference kernels/stream_collide_aa.cu:15-28): in the odd step the
//   thread of node x reads slot (opp i, x - c_i) and writes (i, x + c_i);
//   both belong to x alone, bounce-back slots included. A rule, however,
//   reads populations of other nodes, which the same launch overwrites. The
//   AA kernels therefore never read rule terms from the lattice: every
//   node that a rule term refers to is a SPECIAL exporter whose thread
//   copies f*_k (rounded to the storage format) into export_out after its
//   collision, and the next launch evaluates its rules from that copy
//   (export_in). The two export buffers alternate between launches.
#pragma once

#include <type_traits>

#include "lbm_common.cuh"

namespace lbm {

// Four consecutive reals from a 16-byte aligned address (two loads for double).
__device__ __forceinline__ void load4(const float* p, float (&c)[4])
{
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    c[0] = q.x;
    c[1] = q.y;
    c[2] = q.z;
    c[3] = q.w;
}
__device__ __forceinline__ void load4(const double* p, double (&c)[4])
{
    const double2 q0 = __ldg(reinterpret_cast<const double2*>(p));
    const double2 q1 = __ldg(reinterpret_cast<const double2*>(p + 2));
    c[0] = q0.x;
    c[1] = q0.y;
    c[2] = q1.x;
    c[3] = q1.y;
}

template <class L, int ST, int VAR, int CM = LBM_COLLIDE_TRT>
struct StepKernel {
    using S = Storage<ST>;
    using T = typename S::T;
    using R = typename S::R;
    static constexpr int Q = L::Q;

    // Rule r: const + sum_t coeff[t] f*_{dir[t]}(node[t]), summed in term
    // order with explicit fma. Terms are taken sixteen at a time (a partial
    // last batch is predicated): all term metadata, then all values, so a
    // Zou-He rule -- it combines the 14 known populations of its node --
    // costs two memory round trips instead of two per term.
    __device__ static __forceinline__ R rule_value(const StepArgs& a, int r)
    {
        constexpr int B = 16;
        const lbm_special_t& sp = a.sp;
        const R* __restrict__ coeff = static_cast<const R*>(sp.term_coeff);
        R v = static_cast<const R*>(sp.rule_const)[r];
        const int t1 = sp.term_start[r + 1];
        if (VAR == LBM_PULL) {
            const T* __restrict__ f = static_cast<const T*>(a.f_src);
            for (int t = sp.term_start[r]; t < t1; t += B) {
                int64_t slot[B];
                R c[B], val[B];
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const bool in = t + k < t1;
                    slot[k] = in ? (int64_t)sp.term_dir[t + k] * a.qstride + sp.term_node[t + k] : 0;
                    c[k] = in ? coeff[t + k] : R(0);
                }
#pragma unroll
                for (int k = 0; k < B; ++k) val[k] = S::load(f + slot[k]);
#pragma unroll
                for (int k = 0; k < B; ++k)
                    if (t + k < t1) v = v_fma(c[k], val[k], v);
            }
        } else {
            const R* __restrict__ ex = static_cast<const R*>(sp.export_in);
            for (int t = sp.term_start[r]; t < t1; t += B) {
                int e[B];
                R c[B], val[B];
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const bool in = t + k < t1;
                    e[k] = in ? sp.term_export[t + k] : 0;
                    c[k] = in ? coeff[t + k] : R(0);
                }
#pragma unroll
                for (int k = 0; k < B; ++k) val[k] = ex[e[k]];
#pragma unroll
                for (int k = 0; k < B; ++k)
                    if (t + k < t1) v = v_fma(c[k], val[k], v);
            }
        }
        return v;
    }

    // The node's rules in the dense form (lbm_special_t.ut_start): its distinct
    // term populations are loaded once, all in one batch, then each rule is a
    // dot product with its coefficient row, read four at a time. Two memory
    // round trips for all the node's rules.
    __device__ static __forceinline__ void dense_rules(const StepArgs& a, int64_t s, uint32_t rmask, int rfirst,
                                                       R (&f)[Q])
    {
        constexpr int UM = LBM_DENSE_TERMS;
        const lbm_special_t& sp = a.sp;
        const int u0 = sp.ut_start[s];
        const int n = sp.ut_start[s + 1] - u0;
        R v[UM];
        if (VAR == LBM_PULL) {
            const T* __restrict__ fs = static_cast<const T*>(a.f_src);
            int64_t slot[UM];
#pragma unroll
            for (int u = 0; u < UM; ++u) slot[u] = u < n ? sp.ut_slot[u0 + u] : -1;
#pragma unroll
            for (int u = 0; u < UM; ++u) v[u] = slot[u] >= 0 ? S::load(fs + slot[u]) : R(0);
        } else {
            const R* __restrict__ ex = static_cast<const R*>(sp.export_in);
            int e[UM];
#pragma unroll
            for (int u = 0; u < UM; ++u) e[u] = u < n ? sp.ut_export[u0 + u] : -1;
#pragma unroll
            for (int u = 0; u < UM; ++u) v[u] = e[u] >= 0 ? ex[e[u]] : R(0);
        }
        // the rows of the node's rules are consecutive, (n + 3) & ~3 apart
        const R* __restrict__ row = static_cast<const R*>(sp.rule_dense) + sp.rule_row[rfirst];
        const R* __restrict__ rconst = static_cast<const R*>(sp.rule_const);
        const int n4 = (n + 3) & ~3;
        uint32_t m = rmask;
        int r = rfirst;
        while (m) {
            const int i = __ffs(m) - 1;
            m &= m - 1u;
            R acc = rconst[r++];
#pragma unroll
            for (int u = 0; u < UM; u += 4) {
                if (u < n) {
                    R c[4];
                    load4(row + u, c);
#pragma unroll
                    for (int k = 0; k < 4; ++k) acc = v_fma(c[k], v[u + k], acc);
                }
            }
            row += n4;
#pragma unroll
            for (int j = 0; j < Q; ++j)
                if (j == i) f[j] = acc;
        }
    }

    // Health epilogue of a checked step (pull and AA even: the node's stored
    // values are its post-collision populations): the values as stored,
    // rounded like the stores for 16-bit formats; with a readout, also the
    // node's rho and u from them and the force its collision applied.
    __device__ static __forceinline__ void stored_health(const StepArgs& a, const R (&f)[Q], uint32_t h, bool hi,
                                                         int64_t nd, R Fx, R Fy, R Fz, NodeHealth& hl)
    {
        static_assert(VAR != LBM_AA_ODD, "the odd AA half does not store a node's populations at the node");
        R v[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) v[i] = S::STOCHASTIC ? S::round_sr(f[i], h, i, hi) : f[i];
        health_node<L, R>(hl, nd, v);
        if (a.readout_rho != nullptr)
            store_macro<L, R>(v, Fx, Fy, Fz, nd, a.qstride, static_cast<R*>(a.readout_rho), static_cast<R*>(a.readout_u));
    }

    // Interior fluid node (kind 0: no solid neighbour, not on a face of the
    // box, no rule or local force). Every source and destination offset is
    // the same for all threads (-c_i . strides), so the compiler keeps them in
    // uniform registers and each access is [thread pointer + uniform offset].
    // All Q loads are independent and issued back to back.
    template <bool H = false>
    __device__ static __forceinline__ void interior(const StepArgs& a, int64_t nd, int64_t pair, bool hi,
                                                    NodeHealth* hl = nullptr)
    {
        const int64_t qs = a.qstride;
        const int64_t py = a.pitch;
        const int64_t pz = (int64_t)a.pitch * a.ny;
        R f[Q];
        const T* fs = static_cast<const T*>(a.f_src) + nd;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int64_t shift = L::cx(i) + L::cy(i) * py + L::cz(i) * pz;
            if (VAR == LBM_AA_EVEN)
                f[i] = S::load(fs + i * qs);
            else if (VAR == LBM_PULL)
                f[i] = S::load_nc(fs + (i * qs - shift));
            else
                f[i] = S::load(fs + (L::opp(i) * qs - shift));
        }
        R Fx = R(a.fx), Fy = R(a.fy), Fz = R(a.fz);
        if (a.force_field != nullptr) {
            const R* ff = static_cast<const R*>(a.force_field);
            Fx += ff[nd];
            Fy += ff[qs + nd];
            if (L::D == 3) Fz += ff[2 * qs + nd];
        }
        collide_model<L, R, CM>(f, a.template relax<R>(), a.guo_const && a.force_field == nullptr, Fx, Fy, Fz);
        const uint32_t h = S::STOCHASTIC ? sr_pair_hash(pair, a.seed[a.parity]) : 0u;
        if constexpr (H) stored_health(a, f, h, hi, nd, Fx, Fy, Fz, *hl);
        T* fd = static_cast<T*>(a.f_dst) + nd;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int64_t shift = L::cx(i) + L::cy(i) * py + L::cz(i) * pz;
            if (VAR == LBM_PULL)
                S::store_sr(fd + i * qs, f[i], h, i, hi);
            else if (VAR == LBM_AA_EVEN)
                S::store_sr(fd + L::opp(i) * qs, f[i], h, i, hi);
            else
                S::store_sr(fd + (i * qs + shift), f[i], h, i, hi);
        }
    }

    // General path: bb = solid-neighbour mask (bit i: x - c_i is solid, so
    // bit opp(i): x + c_i is solid). No kind byte of a neighbour is loaded,
    // so all Q loads are independent.
    template <bool SPECIAL, bool H = false>
    __device__ static __forceinline__ void node(const StepArgs& a, int x, int y, int z, int64_t nd, uint32_t bb, int64_t s,
                                                NodeHealth* hl = nullptr)
    {
        const int64_t qs = a.qstride;
        const R* __restrict__ wall = static_cast<const R*>(a.wall_u);
        uint32_t rmask = 0;
        int rfirst = 0;
        if (SPECIAL) {
            rmask = a.sp.rule_mask[s];
            rfirst = a.sp.rule_first[s];
        }
        const int xm = wrap(x - 1, a.nx), xp = wrap(x + 1, a.nx);
        const int ym = wrap(y - 1, a.ny), yp = wrap(y + 1, a.ny);
        const int zm = L::D == 3 ? wrap(z - 1, a.nz) : 0, zp = L::D == 3 ? wrap(z + 1, a.nz) : 0;

        R f[Q];
        // ---- gather the streamed populations
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            if (VAR == LBM_AA_EVEN) {
                f[i] = S::load(static_cast<const T*>(a.f_src) + i * qs + nd);
                continue;
            }
            // source node x - c_i
            const int sx = L::cx(i) > 0 ? xm : (L::cx(i) < 0 ? xp : x);
            const int sy = L::cy(i) > 0 ? ym : (L::cy(i) < 0 ? yp : y);
            const int sz = L::cz(i) > 0 ? zm : (L::cz(i) < 0 ? zp : z);
            const int64_t src = ((int64_t)sz * a.ny + sy) * a.pitch + sx;
            const T* fs = static_cast<const T*>(a.f_src);
            if (i != 0 && ((bb >> i) & 1u)) {
                // halfway bounce-back: the population that left x towards the wall
                const int slot = VAR == LBM_PULL ? L::opp(i) : i;
                f[i] = v_add(S::load(fs + slot * qs + nd), wall_term<L, R>(i, wall, src, qs));
            } else if (VAR == LBM_PULL) {
                f[i] = S::load_nc(fs + i * qs + src);
            } else {
                f[i] = S::load(fs + L::opp(i) * qs + src);
            }
        }

        // ---- link rules replace the bounce-back value of their links. One
        // loop over the set bits keeps a single copy of the term loop; the
        // unrolled select writes the value without indexing f[] at run time.
        if (SPECIAL && rmask) {
            if (a.sp.ut_start != nullptr) {
                dense_rules(a, s, rmask, rfirst, f);
            } else {
                uint32_t m = rmask;
                int r = rfirst;
                while (m) {
                    const int i = __ffs(m) - 1;
                    m &= m - 1u;
                    const R v = rule_value(a, r++);
#pragma unroll
                    for (int j = 0; j < Q; ++j)
                        if (j == i) f[j] = v;
                }
            }
        }

        // ---- collide
        R Fx = R(a.fx), Fy = R(a.fy), Fz = R(a.fz);
        if (a.force_field != nullptr) {
            const R* ff = static_cast<const R*>(a.force_field);
            Fx += ff[nd];
            Fy += ff[qs + nd];
            if (L::D == 3) Fz += ff[2 * qs + nd];
        }
        bool uniform = a.guo_const && a.force_field == nullptr;
        if (SPECIAL) {
            const int fs = a.sp.force_slot[s];
            if (fs >= 0) {
                uniform = false;
                const R* lf = static_cast<const R*>(a.sp.local_force);
                const int64_t n = a.sp.n_local;
                Fx += lf[fs];
                Fy += lf[n + fs];
                if (L::D == 3) Fz += lf[2 * n + fs];
            }
        }
        collide_model<L, R, CM>(f, a.template relax<R>(), uniform, Fx, Fy, Fz);
        const uint32_t h = S::STOCHASTIC ? sr_pair_hash(sr_pair(a.nx, a.ny, x, y, z), a.seed[a.parity]) : 0u;
        const bool hi = x & 1;
        if constexpr (H) stored_health(a, f, h, hi, nd, Fx, Fy, Fz, *hl);

        // ---- store (16-bit formats: stochastic rounding, see sr_pair_hash)
        T* fd = static_cast<T*>(a.f_dst);
        if (VAR == LBM_PULL) {
#pragma unroll
            for (int i = 0; i < Q; ++i) S::store_sr(fd + i * qs + nd, f[i], h, i, hi);
        } else if (VAR == LBM_AA_EVEN) {
#pragma unroll
            for (int i = 0; i < Q; ++i) S::store_sr(fd + L::opp(i) * qs + nd, f[i], h, i, hi);
        } else {
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const int dx = L::cx(i) > 0 ? xp : (L::cx(i) < 0 ? xm : x);
                const int dy = L::cy(i) > 0 ? yp : (L::cy(i) < 0 ? ym : y);
                const int dz = L::cz(i) > 0 ? zp : (L::cz(i) < 0 ? zm : z);
                const int64_t dst = ((int64_t)dz * a.ny + dy) * a.pitch + dx;
                if (i != 0 && ((bb >> L::opp(i)) & 1u)) {
                    S::store_sr(fd + L::opp(i) * qs + nd, v_add(f[i], wall_term<L, R>(L::opp(i), wall, dst, qs)), h, i, hi);
                } else {
                    S::store_sr(fd + i * qs + dst, f[i], h, i, hi);
                }
            }
        }

        // ---- AA rule-term exports
        if (SPECIAL && VAR != LBM_PULL) {
            const uint32_t emask = a.sp.export_mask[s];
            if (emask) {
                R* out = static_cast<R*>(a.sp.export_out);
                int e = a.sp.export_first[s];
                uint32_t m = emask;
                while (m) {
                    const int k = __ffs(m) - 1;
                    m &= m - 1u;
                    R v = f[0];
#pragma unroll
                    for (int j = 1; j < Q; ++j)
                        if (j == k) v = f[j];
                    out[e++] = S::round_sr(v, h, k, hi);
                }
            }
        }
    }
};

// One node of the bulk grid. Every lane of the warp calls it (in = false
// for lanes past the edge of the domain), because the path is chosen per
// warp: a warp whose nodes are all interior (kind 0) takes the branch-free
// path; in any other warp every lane takes the general path (interior lanes
// with an empty mask), so no warp runs both paths one after the other.
// Solid nodes are skipped, SPECIAL nodes are left to the boundary warps.
template <class L, int ST, int VAR, bool H = false, int CM = LBM_COLLIDE_TRT>
__device__ __forceinline__ void bulk_node(const StepArgs& a, int x, int y, int z, int64_t nd, bool in,
                                          NodeHealth* hl = nullptr)
{
    using K = StepKernel<L, ST, VAR, CM>;
    const uint8_t k = in ? a.kind[nd] : KIND_SOLID;
    if (__all_sync(0xffffffffu, !in || k == KIND_FLUID)) {
        if (in) K::template interior<H>(a, nd, sr_pair(a.nx, a.ny, x, y, z), x & 1, hl);
    } else if (!(k & (KIND_SOLID | KIND_SPECIAL))) {
        K::template node<false, H>(a, x, y, z, nd, a.nbr[nd], -1, hl);
    }
}

// Bulk: tile (blockIdx.x, blockIdx.y) of plane z; tile_x is a multiple of
// 32, so every warp lies in one row.
template <class L, int ST, int VAR, bool H = false, int CM = LBM_COLLIDE_TRT>
__device__ __forceinline__ void bulk_tile(const StepArgs& a, int z, NodeHealth* hl = nullptr)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    bulk_node<L, ST, VAR, H, CM>(a, x, y, z, ((int64_t)z * a.ny + y) * a.pitch + x, x < a.nx && y < a.ny, hl);
}

// ---------------------------------------------------------------- vector pull
// Two-lattice pull for 16-bit storage with the two nodes of a pair (x even,
// x + 1) per thread: one 4-byte load and one 4-byte store per direction move
// both populations, the two collisions are independent (instruction-level
// parallelism), and one cvt.rs converts both results with stochastic
// rounding (see sr_pair_hash). A warp covers 64 nodes of one row.
//   * Links along y and z read the aligned pair of the shifted row.
//   * Links along x need the pair shifted by one node: it is rebuilt from the
//     thread's own word and one word of the neighbouring lane (warp shuffle);
//     lanes 0 and 31 load the one node beyond the warp's range themselves,
//     with x wrapped on the periodic faces.
// The vector path runs when every node of the warp's range is interior or on
// a periodic x face (kinds 0 and EDGE, rows off the y and z faces), the
// range lies inside [0, nx) and the force is uniform (the launch picks the
// one-node kernel for per-node force fields); any other warp updates its
// nodes one at a time (bulk_node), lane l taking nodes x_base + 32 k + l so
// that accesses stay coalesced. float16 runs the collision on populations
// times 2^14, which is exact. Per node the arithmetic and the rounding are
// those of the one-node paths: the bits do not depend on the path.
template <class L, int ST>
struct VecPull {
    using S = Storage<ST>;
    using T = typename S::T;
    using R = typename S::R;
    static constexpr int Q = L::Q;
    static constexpr int V = 2;
    static_assert(sizeof(T) == 2, "two 16-bit populations per word");

    __device__ static __forceinline__ void run(const StepArgs& a, int x_base, int y, int z)
    {
        constexpr unsigned FULL = 0xffffffffu;
        const int lane = threadIdx.x & 31;
        const int64_t qs = a.qstride;
        const int64_t py = a.pitch;
        const int64_t pz = (int64_t)a.pitch * a.ny;
        const int64_t row = (int64_t)z * pz + (int64_t)y * py;
        const int x0 = x_base + V * lane;
        const int64_t nd0 = row + x0;
        const bool in_row = y < a.ny;
        bool fast = in_row && x_base + 32 * V <= a.nx && y > 0 && y < a.ny - 1 &&
                    (L::D == 2 || (z > 0 && z < a.nz - 1));
        if (fast) fast = (*reinterpret_cast<const unsigned short*>(a.kind + nd0) & ~0x0808u) == 0u;
        if (!__all_sync(FULL, fast)) {
            for (int j = 0; j < V; ++j) {
                const int x = x_base + 32 * j + lane;
                bulk_node<L, ST, LBM_PULL>(a, x, y, z, row + x, in_row && x < a.nx);
            }
            return;
        }
        // periodic x: the nodes just outside the warp's range
        const int x_lo = x_base == 0 ? a.nx - 1 : x_base - 1;
        const int x_hi = x_base + 32 * V == a.nx ? 0 : x_base + 32 * V;
        const T* fs = static_cast<const T*>(a.f_src);
        R fa[Q], fb[Q];  // the even and the odd node
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int64_t shifted_row = row - (L::cy(i) * py + L::cz(i) * pz) + i * qs;
            const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(fs + shifted_row + x0));
            uint32_t s = w;
            if (L::cx(i) > 0) {  // sources x - 1: (own first, last of lane - 1)
                uint32_t pw = __shfl_up_sync(FULL, w, 1);
                if (lane == 0) pw = (uint32_t)__ldg(reinterpret_cast<const unsigned short*>(fs + shifted_row + x_lo)) << 16;
                s = __byte_perm(pw, w, 0x5432);
            } else if (L::cx(i) < 0) {  // sources x + 1: (first of lane + 1, own last)
                uint32_t nw = __shfl_down_sync(FULL, w, 1);
                if (lane == 31) nw = __ldg(reinterpret_cast<const unsigned short*>(fs + shifted_row + x_hi));
                s = __byte_perm(w, nw, 0x5432);
            }
            fa[i] = S::decode_lo(s);
            fb[i] = S::decode_hi(s);
        }
        const Relax<R>& rc = a.template relax<R>();
        const R Fx = R(a.fx), Fy = R(a.fy), Fz = R(a.fz);
        collide_pair<L, S::SCALE_LOG2>(fa, fb, rc, Fx, Fy, Fz);
        const uint32_t h = sr_pair_hash(sr_pair(a.nx, a.ny, x0, y, z), a.seed[a.parity]);
        T* fd = static_cast<T*>(a.f_dst) + nd0;
#pragma unroll
        for (int i = 0; i < Q; ++i)
            *reinterpret_cast<uint32_t*>(fd + i * qs) = S::pack_sr(fa[i], fb[i], sr_word(h, i));
    }
};

// Vector bulk launch: grid (ceil(nx / (2 tile_x)), ceil(ny / tile_y), nz).
template <class L, int ST>
__global__ void __launch_bounds__(256) lbm_bulk_vec_kernel(const StepArgs a)
{
    advance_seed(a);
    const int warp_x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    VecPull<L, ST>::run(a, warp_x * 64, blockIdx.y * blockDim.y + threadIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------- vector AA
// The in-place AA step for 16-bit storage with node pairs (x even, x + 1)
// per thread, as VecPull: 4-byte loads and stores, two collisions, one
// cvt.rs per direction for both results.
//   * even (node-local): pair i read from slot i, written to slot opp(i) of
//     the same pair -- no neighbour, so any warp without SOLID or SPECIAL
//     nodes takes it (walls and faces do not matter here).
//   * odd: read slot opp(i) of x - c_i (the VecPull gather: x shifts by
//     warp shuffle, the node beyond the warp's range loaded by lane 0 or 31)
//     and write slot i of x + c_i. For c_x != 0 the destination pairs
//     straddle the source pairs: each lane rounds its own two results (its
//     own random word, as the one-node path), then a shuffle hands the half
//     that crosses to the neighbouring lane, which stores the assembled
//     pair; the half leaving the warp's range is stored alone (2 bytes) by
//     lane 0 or 31, and the slot whose source lies outside the range is left
//     to the warp that owns that source. Every slot is written once. Taken
//     by warps of interior nodes (periodic x faces included), rows off the y
//     and z faces.
// Other warps update their nodes one at a time (bulk_node). Same bits as the
// one-node path.
template <class L, int ST, int VAR>
struct VecAA {
    using S = Storage<ST>;
    using T = typename S::T;
    using R = typename S::R;
    static constexpr int Q = L::Q;
    static constexpr int V = 2;
    static_assert(sizeof(T) == 2, "two 16-bit populations per word");
    static_assert(VAR == LBM_AA_EVEN || VAR == LBM_AA_ODD, "AA halves only");

    __device__ static __forceinline__ void run(const StepArgs& a, int x_base, int y, int z)
    {
        constexpr unsigned FULL = 0xffffffffu;
        const int lane = threadIdx.x & 31;
        const int64_t qs = a.qstride;
        const int64_t py = a.pitch;
        const int64_t pz = (int64_t)a.pitch * a.ny;
        const int64_t row = (int64_t)z * pz + (int64_t)y * py;
        const int x0 = x_base + V * lane;
        const int64_t nd0 = row + x0;
        const bool in_row = y < a.ny;
        bool fast = in_row && x_base + 32 * V <= a.nx;
        if (VAR == LBM_AA_ODD) fast = fast && y > 0 && y < a.ny - 1 && (L::D == 2 || (z > 0 && z < a.nz - 1));
        if (fast) {
            const uint32_t k2 = *reinterpret_cast<const unsigned short*>(a.kind + nd0);
            fast = VAR == LBM_AA_EVEN ? (k2 & 0x0303u) == 0u : (k2 & ~0x0808u) == 0u;
        }
        if (!__all_sync(FULL, fast)) {
            for (int j = 0; j < V; ++j) {
                const int x = x_base + 32 * j + lane;
                bulk_node<L, ST, VAR>(a, x, y, z, row + x, in_row && x < a.nx);
            }
            return;
        }
        // periodic x: the nodes just outside the warp's range
        const int x_lo = x_base == 0 ? a.nx - 1 : x_base - 1;
        const int x_hi = x_base + 32 * V == a.nx ? 0 : x_base + 32 * V;
        T* f = static_cast<T*>(a.f_dst);  // in place: f_src == f_dst
        R fa[Q], fb[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            uint32_t s;
            if (VAR == LBM_AA_EVEN) {
                s = *reinterpret_cast<const uint32_t*>(f + i * qs + nd0);
            } else {
                const int64_t src_row = row - (L::cy(i) * py + L::cz(i) * pz) + L::opp(i) * qs;
                const uint32_t w = *reinterpret_cast<const uint32_t*>(f + src_row + x0);
                s = w;
                if (L::cx(i) > 0) {  // sources x - 1
                    uint32_t pw = __shfl_up_sync(FULL, w, 1);
                    if (lane == 0) pw = (uint32_t)*reinterpret_cast<const unsigned short*>(f + src_row + x_lo) << 16;
                    s = __byte_perm(pw, w, 0x5432);
                } else if (L::cx(i) < 0) {  // sources x + 1
                    uint32_t nw = __shfl_down_sync(FULL, w, 1);
                    if (lane == 31) nw = *reinterpret_cast<const unsigned short*>(f + src_row + x_hi);
                    s = __byte_perm(w, nw, 0x5432);
                }
            }
            fa[i] = S::decode_lo(s);
            fb[i] = S::decode_hi(s);
        }
        const Relax<R>& rc = a.template relax<R>();
        const R Fx = R(a.fx), Fy = R(a.fy), Fz = R(a.fz);
        collide_pair<L, S::SCALE_LOG2>(fa, fb, rc, Fx, Fy, Fz);
        const uint32_t h = sr_pair_hash(sr_pair(a.nx, a.ny, x0, y, z), a.seed[a.parity]);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const uint32_t w = S::pack_sr(fa[i], fb[i], sr_word(h, i));  // (x0, x0 + 1) rounded
            if (VAR == LBM_AA_EVEN) {
                *reinterpret_cast<uint32_t*>(f + L::opp(i) * qs + nd0) = w;
                continue;
            }
            T* dst_row = f + i * qs + row + (L::cy(i) * py + L::cz(i) * pz);
            if (L::cx(i) == 0) {
                *reinterpret_cast<uint32_t*>(dst_row + x0) = w;
            } else if (L::cx(i) > 0) {  // x -> x + 1: pair (x0, x0 + 1) <- (lane - 1's odd node, own even node)
                const uint32_t pw = __shfl_up_sync(FULL, w, 1);
                if (lane == 0)
                    *reinterpret_cast<unsigned short*>(dst_row + x0 + 1) = (unsigned short)(w & 0xffffu);
                else
                    *reinterpret_cast<uint32_t*>(dst_row + x0) = __byte_perm(pw, w, 0x5432);
                if (lane == 31) *reinterpret_cast<unsigned short*>(dst_row + x_hi) = (unsigned short)(w >> 16);
            } else {  // x -> x - 1: pair (x0, x0 + 1) <- (own odd node, lane + 1's even node)
                const uint32_t nw = __shfl_down_sync(FULL, w, 1);
                if (lane == 31)
                    *reinterpret_cast<unsigned short*>(dst_row + x0) = (unsigned short)(w >> 16);
                else
                    *reinterpret_cast<uint32_t*>(dst_row + x0) = __byte_perm(w, nw, 0x5432);
                if (lane == 0) *reinterpret_cast<unsigned short*>(dst_row + x_lo) = (unsigned short)(w & 0xffffu);
            }
        }
    }
};

template <class L, int ST, int VAR>
__global__ void __launch_bounds__(256) lbm_bulk_vec_aa_kernel(const StepArgs a)
{
    advance_seed(a);
    const int warp_x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    VecAA<L, ST, VAR>::run(a, warp_x * 64, blockIdx.y * blockDim.y + threadIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------- odd AA, rows
// The odd AA half for float32/float64 with one block per row (nx <= 256):
// a row whose nodes are all interior in y and z (kinds 0 and EDGE, the row off
// the y and z faces) pulls and collides each node as the interior path does
// (x wrapped in the row), writes its results into shared memory in
// destination order -- f*_i of node x at x + c_x, wrapped -- and then stores
// every direction's destination row (y + c_y, z + c_z) whole, each thread one
// aligned element: the pushes along x no longer store to rows shifted by one
// element, which half-fill 32-byte sectors that other warps complete. Other
// rows run the one-node path (bulk_node). Same bits as the one-node kernel.
// In place is safe: slot i of row (y + c_y, z + c_z) is read, in this half,
// only by the nodes of row (y, z) -- this block -- before the block's barrier.
// With the TRT collision, a bound on the registers keeps more rows' loads in
// flight than ptxas's own choice (the one-node fallback spills a little):
// 4-byte storage six 256-thread blocks per SM (40 registers; ptxas alone: 64,
// four blocks), 39.8 against 37.4 GLUPS for the AA pair on the 256^3 duct
// (seven blocks, 32 registers: slower); 8-byte storage three blocks
// (80 registers; alone: 102, two blocks), 21.4 against 19.9 GLUPS.
template <int ST, int CM>
constexpr int odd_rows_min_blocks()
{
    if (CM != LBM_COLLIDE_TRT) return 0;
    return sizeof(typename Storage<ST>::T) == 4 ? 6 : 3;
}

template <class L, int ST, int CM>
__global__ void __launch_bounds__(256, odd_rows_min_blocks<ST, CM>()) lbm_aa_odd_rows_kernel(const StepArgs a)
{
    using S = Storage<ST>;
    using T = typename S::T;
    using R = typename S::R;
    constexpr int Q = L::Q;
    extern __shared__ __align__(16) unsigned char rows_smem[];
    T* out = reinterpret_cast<T*>(rows_smem);
    advance_seed(a);
    const int nx = a.nx, y = blockIdx.x, z = blockIdx.y, x = threadIdx.x;
    const bool in = x < nx;
    const int64_t py = a.pitch, pz = (int64_t)a.pitch * a.ny, qs = a.qstride;
    const int64_t row = (int64_t)z * pz + (int64_t)y * py;
    const int64_t nd = row + x;
    const uint8_t k = in ? a.kind[nd] : KIND_FLUID;
    const bool row_ok = y >= 1 && y <= a.ny - 2 && (L::D == 2 || (z >= 1 && z <= a.nz - 2));
    if (!__syncthreads_and(row_ok && (k & ~KIND_EDGE) == 0)) {
        bulk_node<L, ST, LBM_AA_ODD, false, CM>(a, x, y, z, nd, in);
        return;
    }
    if (in) {
        const int xm = x == 0 ? nx - 1 : x - 1, xp = x + 1 == nx ? 0 : x + 1;
        const T* f = static_cast<const T*>(a.f_src);
        R fv[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int sx = L::cx(i) > 0 ? xm : (L::cx(i) < 0 ? xp : x);
            fv[i] = S::load(f + (L::opp(i) * qs + row - (L::cy(i) * py + L::cz(i) * pz) + sx));
        }
        R Fx = R(a.fx), Fy = R(a.fy), Fz = R(a.fz);
        if (a.force_field != nullptr) {
            const R* ff = static_cast<const R*>(a.force_field);
            Fx += ff[nd];
            Fy += ff[qs + nd];
            if (L::D == 3) Fz += ff[2 * qs + nd];
        }
        collide_model<L, R, CM>(fv, a.template relax<R>(), a.guo_const && a.force_field == nullptr, Fx, Fy, Fz);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int dx = L::cx(i) > 0 ? xp : (L::cx(i) < 0 ? xm : x);
            out[i * nx + dx] = S::encode(fv[i]);
        }
    }
    __syncthreads();
    if (in) {
        T* f = static_cast<T*>(a.f_dst);
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i * qs + row + (L::cy(i) * py + L::cz(i) * pz) + x] = out[i * nx + x];
    }
}

// ---------------------------------------------------------------- odd AA, rows, 16-bit
// The odd AA half for 16-bit storage with one block per row (nx even, at
// most 256: 128 threads), each thread a node pair (x0, x0 + 1): a row whose nodes are all
// interior in y and z (kinds 0 and EDGE, the row off the y and z faces) reads
// each direction's source pair words from row (y - c_y, z - c_z) of slot
// opp(i) -- the pair's own word, and the neighbouring pair's word for
// directions with c_x != 0 (x wrapped in the row) -- collides the pair as the
// other pair kernels do, rounds it, writes its results into shared memory in
// destination order (x + c_x, wrapped) and, after one barrier, stores every
// destination row (y + c_y, z + c_z) of slot i as aligned pair words. Other
// rows run the one-node path. Same bits as every other kernel of the step;
// in place is safe as in the 4- and 8-byte row kernel: slot i of row
// (y + c_y, z + c_z) is read in this half only by the nodes of row (y, z).
template <class L, int ST>
__global__ void __launch_bounds__(128, 6) lbm_aa_odd_pair_rows_kernel(const StepArgs a)
{
    using S = Storage<ST>;
    using T = typename S::T;
    using R = typename S::R;
    constexpr int Q = L::Q;
    static_assert(sizeof(T) == 2, "two 16-bit populations per word");
    extern __shared__ __align__(16) unsigned char pair_rows_smem[];
    unsigned short* out = reinterpret_cast<unsigned short*>(pair_rows_smem);  // [Q][nx]
    advance_seed(a);
    const int nx = a.nx, y = blockIdx.x, z = blockIdx.y;
    const int x0 = 2 * threadIdx.x;
    const bool in = x0 < nx;
    const int64_t py = a.pitch, pz = (int64_t)a.pitch * a.ny, qs = a.qstride;
    const int64_t row = (int64_t)z * pz + (int64_t)y * py;
    const int64_t nd0 = row + x0;
    const uint32_t k2 = in ? *reinterpret_cast<const unsigned short*>(a.kind + nd0) : 0u;
    const bool row_ok = y >= 1 && y <= a.ny - 2 && (L::D == 2 || (z >= 1 && z <= a.nz - 2));
    if (!__syncthreads_and(row_ok && (k2 & ~0x0808u) == 0u)) {
        for (int h = 0; h < 2; ++h) bulk_node<L, ST, LBM_AA_ODD>(a, x0 + h, y, z, nd0 + h, in);
        return;
    }
    if (in) {
        const int wm = (x0 == 0 ? nx - 2 : x0 - 2) >> 1;  // the previous pair's word, wrapped
        const int wo = x0 >> 1;
        const int wn = (x0 + 2 == nx ? 0 : x0 + 2) >> 1;  // the next pair's word, wrapped
        const unsigned short* fs = static_cast<const unsigned short*>(a.f_src);
        R fa[Q], fb[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(
                fs + (L::opp(i) * qs + row - (L::cy(i) * py + L::cz(i) * pz)));
            if (L::cx(i) == 0) {
                const uint32_t v = w[wo];
                fa[i] = S::decode_lo(v);
                fb[i] = S::decode_hi(v);
            } else if (L::cx(i) > 0) {  // sources x0 - 1, x0
                fa[i] = S::decode_hi(w[wm]);
                fb[i] = S::decode_lo(w[wo]);
            } else {  // sources x0 + 1, x0 + 2
                fa[i] = S::decode_hi(w[wo]);
                fb[i] = S::decode_lo(w[wn]);
            }
        }
        collide_pair<L, S::SCALE_LOG2>(fa, fb, a.template relax<R>(), R(a.fx), R(a.fy), R(a.fz));
        const uint32_t h = sr_pair_hash(sr_pair(nx, a.ny, x0, y, z), a.seed[a.parity]);
        const int xm = x0 == 0 ? nx - 1 : x0 - 1;
        const int xp = x0 + 2 == nx ? 0 : x0 + 2;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const uint32_t v = S::pack_sr(fa[i], fb[i], sr_word(h, i));  // (x0, x0 + 1) rounded
            unsigned short* o = out + i * nx;
            if (L::cx(i) == 0) {
                *reinterpret_cast<uint32_t*>(o + x0) = v;
            } else if (L::cx(i) > 0) {  // x0 -> x0 + 1, x0 + 1 -> x0 + 2
                o[x0 + 1] = (unsigned short)v;
                o[xp] = (unsigned short)(v >> 16);
            } else {  // x0 -> x0 - 1, x0 + 1 -> x0
                o[xm] = (unsigned short)v;
                o[x0] = (unsigned short)(v >> 16);
            }
        }
    }
    __syncthreads();
    if (in) {
        T* f = static_cast<T*>(a.f_dst);
#pragma unroll
        for (int i = 0; i < Q; ++i)
            *reinterpret_cast<uint32_t*>(f + (i * qs + row + (L::cy(i) * py + L::cz(i) * pz) + x0)) =
                *reinterpret_cast<const uint32_t*>(out + i * nx + x0);
    }
}

// The two-lattice pull (VAR = LBM_PULL) and the even AA half (LBM_AA_EVEN)
// for 16-bit storage on widths the TMA kernel does not take, one block per
// row (nx even, at most 256), each thread a node pair: a row whose nodes are
// all interior in y and z (kinds 0 and EDGE, the row off the y and z faces)
// reads each direction's pair words -- pull: from row (y - c_y, z - c_z) of
// slot i, the pair's own word and, for directions with c_x != 0, the
// neighbouring pair's word (x wrapped in the row); even AA half: the pair's
// own word of slot i -- collides the pair as the other pair kernels do and
// stores aligned pair words (pull: slot i; even AA half: slot opp(i), in
// place, node-local). No warp straddles two rows, so no row falls back for
// that; rows with other nodes run the one-node path. Same bits as every other
// kernel of the step.
template <class L, int ST, int VAR>
__global__ void __launch_bounds__(128, 6) lbm_pair_rows_kernel(const StepArgs a)
{
    using S = Storage<ST>;
    using T = typename S::T;
    using R = typename S::R;
    constexpr int Q = L::Q;
    static_assert(sizeof(T) == 2, "two 16-bit populations per word");
    advance_seed(a);
    const int nx = a.nx, y = blockIdx.x, z = blockIdx.y;
    const int x0 = 2 * threadIdx.x;
    const bool in = x0 < nx;
    const int64_t py = a.pitch, pz = (int64_t)a.pitch * a.ny, qs = a.qstride;
    const int64_t row = (int64_t)z * pz + (int64_t)y * py;
    const int64_t nd0 = row + x0;
    const uint32_t k2 = in ? *reinterpret_cast<const unsigned short*>(a.kind + nd0) : 0u;
    const bool row_ok = y >= 1 && y <= a.ny - 2 && (L::D == 2 || (z >= 1 && z <= a.nz - 2));
    if (!__syncthreads_and(row_ok && (k2 & ~0x0808u) == 0u)) {
        for (int h = 0; h < 2; ++h) bulk_node<L, ST, VAR>(a, x0 + h, y, z, nd0 + h, in);
        return;
    }
    if (!in) return;
    const int wm = (x0 == 0 ? nx - 2 : x0 - 2) >> 1;  // the previous pair's word, wrapped
    const int wo = x0 >> 1;
    const int wn = (x0 + 2 == nx ? 0 : x0 + 2) >> 1;  // the next pair's word, wrapped
    const unsigned short* fs = static_cast<const unsigned short*>(a.f_src);
    R fa[Q], fb[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        if constexpr (VAR == LBM_AA_EVEN) {  // node-local, in place: plain loads
            const uint32_t v = *reinterpret_cast<const uint32_t*>(fs + (i * qs + nd0));
            fa[i] = S::decode_lo(v);
            fb[i] = S::decode_hi(v);
            continue;
        }
        const uint32_t* w = reinterpret_cast<const uint32_t*>(fs + (i * qs + row - (L::cy(i) * py + L::cz(i) * pz)));
        if (L::cx(i) == 0) {
            const uint32_t v = __ldg(w + wo);
            fa[i] = S::decode_lo(v);
            fb[i] = S::decode_hi(v);
        } else if (L::cx(i) > 0) {  // sources x0 - 1, x0
            fa[i] = S::decode_hi(__ldg(w + wm));
            fb[i] = S::decode_lo(__ldg(w + wo));
        } else {  // sources x0 + 1, x0 + 2
            fa[i] = S::decode_hi(__ldg(w + wo));
            fb[i] = S::decode_lo(__ldg(w + wn));
        }
    }
    collide_pair<L, S::SCALE_LOG2>(fa, fb, a.template relax<R>(), R(a.fx), R(a.fy), R(a.fz));
    const uint32_t h = sr_pair_hash(sr_pair(nx, a.ny, x0, y, z), a.seed[a.parity]);
    T* fd = static_cast<T*>(a.f_dst) + nd0;
#pragma unroll
    for (int i = 0; i < Q; ++i)
        *reinterpret_cast<uint32_t*>(fd + (VAR == LBM_AA_EVEN ? L::opp(i) : i) * qs) =
            S::pack_sr(fa[i], fb[i], sr_word(h, i));
}

// Storage formats with the pair and TMA kernels (float32 and float64 keep
// the one-node kernel: it is faster there).
template <int ST> constexpr bool has_vec() { return ST == LBM_F16 || ST == LBM_BF16; }

}  // namespace lbm

#include "tma_pull.cuh"

namespace lbm {

template <class L, int ST, int VAR, bool H = false, int CM = LBM_COLLIDE_TRT>
__device__ __forceinline__ void boundary_node(const StepArgs& a, int64_t s, NodeHealth* hl = nullptr)
{
    if (s >= a.sp.n_special) return;
    const int64_t nd = a.sp.node[s];
    const int64_t row = nd / a.pitch;
    const int x = (int)(nd - row * a.pitch);
    const int y = (int)(row % a.ny);
    const int z = (int)(row / a.ny);
    StepKernel<L, ST, VAR, CM>::template node<true, H>(a, x, y, z, nd, a.nbr[nd], s, hl);
}

// Bulk-only launches -- this kernel carries almost all of the traffic, so
// its register count sets the resident warps. ptxas's default target is
// kept except where a bound does better without spills: the odd AA half
// (wrapped reads and wrapped writes on its general path) would take 74
// registers in float32 arithmetic, four 256-thread blocks per SM cap it at
// 64 (32 resident warps instead of 24); the float32 pull would take 54, five
// blocks cap it at 48 (40 warps instead of 36: 38.7 against 37.8 GLUPS).
// The checked-step form (H: health epilogue, one step per chunk) keeps the
// default target.
template <int ST, int VAR, bool H = false>
constexpr int bulk_min_blocks()
{
    if (H) return 0;
    if (VAR == LBM_AA_ODD && sizeof(typename Storage<ST>::R) == 4) return 4;
    if (VAR == LBM_PULL && ST == LBM_F32) return 5;
    return 0;
}

template <class L, int ST, int VAR, bool H = false, int CM = LBM_COLLIDE_TRT>
__global__ void __launch_bounds__(256, bulk_min_blocks<ST, VAR, H || CM != LBM_COLLIDE_TRT>()) lbm_bulk_kernel(const StepArgs a)
{
    advance_seed(a);
    if constexpr (H) {
        NodeHealth hl;
        bulk_tile<L, ST, VAR, true, CM>(a, blockIdx.z, &hl);
        health_block(a, hl, ((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
    } else {
        bulk_tile<L, ST, VAR, false, CM>(a, blockIdx.z);
    }
}

// D2Q9 float32 pull on planes far beyond L2 (at least WIDE_PLANE_NODES
// nodes): a D2Q9 node has only nine loads to hide the memory latency with,
// so a bound of eight blocks per SM (32 registers, a small spill on the
// general path) keeps more of them in flight: 2048^2 78.2 against 74.3 GLUPS,
// 4096^2 84.8 against 77.3. Small grids (the cylinder channel, L2-resident
// lattices) keep the default kernel, which is faster there. Same code, so
// the same bits.
constexpr int64_t WIDE_PLANE_NODES = int64_t(1) << 21;

template <class L, int ST>
__global__ void __launch_bounds__(256, 8) lbm_bulk_wide_kernel(const StepArgs a)
{
    advance_seed(a);
    bulk_tile<L, ST, LBM_PULL, false, LBM_COLLIDE_TRT>(a, blockIdx.z);
}

// FUSED: grid (ceil(nx/bx), ceil(ny/by), nz + extra), planes z >= nz are
// boundary warps. BOUNDARY: 1D grid over the list. Up to 255 registers, so
// the general per-node path never spills.
template <class L, int ST, int VAR, int MODE, bool H = false, int CM = LBM_COLLIDE_TRT>
__global__ void __launch_bounds__(256, 1) lbm_step_kernel(const StepArgs a)
{
    NodeHealth hl;
    if (MODE == LBM_LAUNCH_BOUNDARY) {
        boundary_node<L, ST, VAR, H, CM>(a, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, &hl);
        if constexpr (H) health_block(a, hl, blockIdx.x);
        return;
    }
    const int z = blockIdx.z;
    if (z < a.nz) {
        advance_seed(a);
        bulk_tile<L, ST, VAR, H, CM>(a, z, &hl);
    } else {
        const int64_t b = ((int64_t)(z - a.nz) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        boundary_node<L, ST, VAR, H, CM>(a, b * (blockDim.x * blockDim.y) + threadIdx.y * blockDim.x + threadIdx.x, &hl);
    }
    if constexpr (H) health_block(a, hl, ((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
}

// Boundary launches: one warp per block (BOUNDARY_THREADS), so that a few
// thousand special nodes -- each a long chain of dependent loads (rule terms)
// -- spread over every SM instead of filling a few (256-thread blocks put an
// 8,900-node list on 35 of the 148 SMs).

// A checked step (health epilogue): the one-node bulk kernel, whatever the
// storage (every bulk kernel gives the same bits), and boundary warps whose
// per-block sums follow the bulk grid's in the partial array.
template <class L, int ST, int VAR, int CM>
static int launch_checked(StepArgs a, int mode, int tile_x, int tile_y, cudaStream_t stream)
{
    if constexpr (VAR == LBM_AA_ODD) {
        return LBM_ERR_INVALID;
    } else {
        const unsigned gx = (unsigned)((a.nx + tile_x - 1) / tile_x);
        const unsigned gy = (unsigned)((a.ny + tile_y - 1) / tile_y);
        if (mode == LBM_LAUNCH_BOUNDARY) {
            if (a.sp.n_special <= 0) return LBM_OK;
            a.health_slot0 = (int64_t)gx * gy * a.nz;
            const int64_t blocks = (a.sp.n_special + BOUNDARY_THREADS - 1) / BOUNDARY_THREADS;
            lbm_step_kernel<L, ST, VAR, LBM_LAUNCH_BOUNDARY, true, CM><<<(unsigned)blocks, BOUNDARY_THREADS, 0, stream>>>(a);
        } else if (mode == LBM_LAUNCH_BULK) {
            if (a.nz > 65535) return LBM_ERR_INVALID;
            a.health_slot0 = 0;
            lbm_bulk_kernel<L, ST, VAR, true, CM><<<dim3(gx, gy, a.nz), dim3(tile_x, tile_y), 0, stream>>>(a);
        } else {
            const int64_t per_plane = (int64_t)gx * gy * tile_x * tile_y;
            const int64_t extra = a.sp.n_special > 0 ? (a.sp.n_special + per_plane - 1) / per_plane : 0;
            if (a.nz + extra > 65535) return LBM_ERR_INVALID;
            a.health_slot0 = 0;
            lbm_step_kernel<L, ST, VAR, LBM_LAUNCH_FUSED, true, CM>
                <<<dim3(gx, gy, (unsigned)(a.nz + extra)), dim3(tile_x, tile_y), 0, stream>>>(a);
        }
        return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
    }
}

// CM: the collision model; the node-pair and TMA-staged kernels implement
// TRT/BGK only, so another model takes the one-node kernels.
template <class L, int ST, int VAR, int CM = LBM_COLLIDE_TRT>
static int launch_mode(const StepArgs& a, int mode, int tile_x, int tile_y, cudaStream_t stream)
{
    if (a.health_words != nullptr) return launch_checked<L, ST, VAR, CM>(a, mode, tile_x, tile_y, stream);
    const int threads = tile_x * tile_y;
    const unsigned gx = (unsigned)((a.nx + tile_x - 1) / tile_x);
    const unsigned gy = (unsigned)((a.ny + tile_y - 1) / tile_y);
    if (mode == LBM_LAUNCH_BOUNDARY) {
        if (a.sp.n_special <= 0) return LBM_OK;
        const int64_t blocks = (a.sp.n_special + BOUNDARY_THREADS - 1) / BOUNDARY_THREADS;
        lbm_step_kernel<L, ST, VAR, LBM_LAUNCH_BOUNDARY, false, CM><<<(unsigned)blocks, BOUNDARY_THREADS, 0, stream>>>(a);
    } else if (mode == LBM_LAUNCH_BULK) {
        if (a.nz > 65535) return LBM_ERR_INVALID;
        if constexpr (VAR == LBM_PULL && has_vec<ST>() && CM == LBM_COLLIDE_TRT) {
            int status = LBM_OK;
            if (launch_tma<L, ST, LBM_PULL>(a, stream, &status)) return status;
            // widths the TMA kernel does not take: one block per row
            if (a.nx % 2 == 0 && a.nx <= 2 * 128 && a.ny <= 65535 && a.pitch % 2 == 0 && a.qstride % 2 == 0 &&
                a.force_field == nullptr && a.guo_const && a.seed != nullptr &&
                reinterpret_cast<uintptr_t>(a.kind) % 2 == 0 && reinterpret_cast<uintptr_t>(a.f_src) % 4 == 0 &&
                reinterpret_cast<uintptr_t>(a.f_dst) % 4 == 0) {
                const unsigned threads = (unsigned)((a.nx / 2 + 31) / 32 * 32);
                lbm_pair_rows_kernel<L, ST, LBM_PULL><<<dim3((unsigned)a.ny, (unsigned)a.nz), threads, 0, stream>>>(a);
                return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
            }
            // pairs need every row and direction plane to start on an even
            // node, and the launch's uniform-force constants
            if (a.pitch % 2 == 0 && a.qstride % 2 == 0 && a.force_field == nullptr && a.guo_const) {
                const unsigned gxv = (unsigned)((a.nx + 2 * tile_x - 1) / (2 * tile_x));
                lbm_bulk_vec_kernel<L, ST><<<dim3(gxv, gy, a.nz), dim3(tile_x, tile_y), 0, stream>>>(a);
                return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
            }
        }
        if constexpr (VAR == LBM_AA_ODD && !has_vec<ST>()) {
            if (a.nx <= 256 && a.ny <= 65535) {
                const unsigned threads = (unsigned)((a.nx + 31) / 32 * 32);
                const size_t smem = (size_t)L::Q * a.nx * sizeof(typename Storage<ST>::T);
                lbm_aa_odd_rows_kernel<L, ST, CM><<<dim3((unsigned)a.ny, (unsigned)a.nz), threads, smem, stream>>>(a);
                return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
            }
        }
        if constexpr (VAR != LBM_PULL && has_vec<ST>() && CM == LBM_COLLIDE_TRT) {
            int status = LBM_OK;
            if (launch_tma<L, ST, VAR>(a, stream, &status)) return status;
            // the odd half on widths the TMA kernel does not take: one block per row (same speed
            // as the TMA kernel where both apply); the even half likewise
            if constexpr (VAR == LBM_AA_EVEN) {
                if (a.nx % 2 == 0 && a.nx <= 2 * 128 && a.ny <= 65535 && a.pitch % 2 == 0 && a.qstride % 2 == 0 &&
                    a.force_field == nullptr && a.guo_const && a.seed != nullptr &&
                    reinterpret_cast<uintptr_t>(a.kind) % 2 == 0 && reinterpret_cast<uintptr_t>(a.f_src) % 4 == 0 &&
                    reinterpret_cast<uintptr_t>(a.f_dst) % 4 == 0) {
                    const unsigned threads = (unsigned)((a.nx / 2 + 31) / 32 * 32);
                    lbm_pair_rows_kernel<L, ST, LBM_AA_EVEN><<<dim3((unsigned)a.ny, (unsigned)a.nz), threads, 0, stream>>>(a);
                    return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
                }
            }
            if constexpr (VAR == LBM_AA_ODD) {
                if (a.nx % 2 == 0 && a.nx <= 2 * 128 && a.ny <= 65535 && a.pitch % 2 == 0 && a.qstride % 2 == 0 &&
                    a.force_field == nullptr && a.guo_const && a.seed != nullptr &&
                    reinterpret_cast<uintptr_t>(a.kind) % 2 == 0 && reinterpret_cast<uintptr_t>(a.f_src) % 4 == 0 &&
                    reinterpret_cast<uintptr_t>(a.f_dst) % 4 == 0) {
                    const unsigned threads = (unsigned)((a.nx / 2 + 31) / 32 * 32);
                    const size_t smem = (size_t)L::Q * a.nx * sizeof(typename Storage<ST>::T);
                    lbm_aa_odd_pair_rows_kernel<L, ST><<<dim3((unsigned)a.ny, (unsigned)a.nz), threads, smem, stream>>>(a);
                    return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
                }
            }
            // node pairs: every row and direction plane starts on an even node
            if (a.pitch % 2 == 0 && a.qstride % 2 == 0 && a.force_field == nullptr && a.guo_const) {
                const unsigned gxv = (unsigned)((a.nx + 2 * tile_x - 1) / (2 * tile_x));
                lbm_bulk_vec_aa_kernel<L, ST, VAR><<<dim3(gxv, gy, a.nz), dim3(tile_x, tile_y), 0, stream>>>(a);
                return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
            }
        }
        if constexpr (L::D == 2 && ST == LBM_F32 && VAR == LBM_PULL && CM == LBM_COLLIDE_TRT) {
            if ((int64_t)a.nx * a.ny >= WIDE_PLANE_NODES) {
                lbm_bulk_wide_kernel<L, ST><<<dim3(gx, gy, a.nz), dim3(tile_x, tile_y), 0, stream>>>(a);
                return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
            }
        }
        lbm_bulk_kernel<L, ST, VAR, false, CM><<<dim3(gx, gy, a.nz), dim3(tile_x, tile_y), 0, stream>>>(a);
    } else {
        const int64_t per_plane = (int64_t)gx * gy * threads;
        const int64_t extra = a.sp.n_special > 0 ? (a.sp.n_special + per_plane - 1) / per_plane : 0;
        if (a.nz + extra > 65535) return LBM_ERR_INVALID;
        lbm_step_kernel<L, ST, VAR, LBM_LAUNCH_FUSED, false, CM>
            <<<dim3(gx, gy, (unsigned)(a.nz + extra)), dim3(tile_x, tile_y), 0, stream>>>(a);
    }
    return cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
}

template <class L, int ST>
int launch_step(const StepArgs& a, int variant, int mode, int tile_x, int tile_y, cudaStream_t stream)
{
    if (mode < LBM_LAUNCH_FUSED || mode > LBM_LAUNCH_BOUNDARY) return LBM_ERR_INVALID;
    if (a.collision == LBM_COLLIDE_REGULARIZED) {
        switch (variant) {
        case LBM_PULL: return launch_mode<L, ST, LBM_PULL, LBM_COLLIDE_REGULARIZED>(a, mode, tile_x, tile_y, stream);
        case LBM_AA_EVEN: return launch_mode<L, ST, LBM_AA_EVEN, LBM_COLLIDE_REGULARIZED>(a, mode, tile_x, tile_y, stream);
        case LBM_AA_ODD: return launch_mode<L, ST, LBM_AA_ODD, LBM_COLLIDE_REGULARIZED>(a, mode, tile_x, tile_y, stream);
        default: return LBM_ERR_INVALID;
        }
    }
    if (a.collision == LBM_COLLIDE_CUMULANT) {
        if constexpr (L::D == 2) {
            switch (variant) {
            case LBM_PULL: return launch_mode<L, ST, LBM_PULL, LBM_COLLIDE_CUMULANT>(a, mode, tile_x, tile_y, stream);
            case LBM_AA_EVEN: return launch_mode<L, ST, LBM_AA_EVEN, LBM_COLLIDE_CUMULANT>(a, mode, tile_x, tile_y, stream);
            case LBM_AA_ODD: return launch_mode<L, ST, LBM_AA_ODD, LBM_COLLIDE_CUMULANT>(a, mode, tile_x, tile_y, stream);
            default: return LBM_ERR_INVALID;
            }
        }
        return LBM_ERR_UNSUPPORTED;  // D2Q9 only
    }
    if (a.collision != LBM_COLLIDE_TRT) return LBM_ERR_INVALID;
    switch (variant) {
    case LBM_PULL: return launch_mode<L, ST, LBM_PULL>(a, mode, tile_x, tile_y, stream);
    case LBM_AA_EVEN: return launch_mode<L, ST, LBM_AA_EVEN>(a, mode, tile_x, tile_y, stream);
    case LBM_AA_ODD: return launch_mode<L, ST, LBM_AA_ODD>(a, mode, tile_x, tile_y, stream);
    default: return LBM_ERR_INVALID;
    }
}

template <class L, int ST, int VAR>
static cudaError_t attrs(cudaFuncAttributes* attr, int mode)
{
    switch (mode) {
    case LBM_LAUNCH_FUSED: return cudaFuncGetAttributes(attr, lbm_step_kernel<L, ST, VAR, LBM_LAUNCH_FUSED>);
    case LBM_LAUNCH_BULK: return cudaFuncGetAttributes(attr, lbm_bulk_kernel<L, ST, VAR>);
    default: return cudaFuncGetAttributes(attr, lbm_step_kernel<L, ST, VAR, LBM_LAUNCH_BOUNDARY>);
    }
}

// which = variant + 3 * mode
template <class L, int ST>
int step_resources(int which, int32_t* out4)
{
    cudaFuncAttributes attr;
    cudaError_t e;
    const int variant = which % 3, mode = which / 3;
    if (mode > LBM_LAUNCH_BOUNDARY || which < 0) return LBM_ERR_INVALID;
    switch (variant) {
    case LBM_PULL: e = attrs<L, ST, LBM_PULL>(&attr, mode); break;
    case LBM_AA_EVEN: e = attrs<L, ST, LBM_AA_EVEN>(&attr, mode); break;
    default: e = attrs<L, ST, LBM_AA_ODD>(&attr, mode); break;
    }
    if (e != cudaSuccess) return LBM_ERR_LAUNCH;
    out4[0] = attr.numRegs;
    out4[1] = (int32_t)attr.localSizeBytes;
    out4[2] = (int32_t)attr.sharedSizeBytes;
    out4[3] = attr.maxThreadsPerBlock;
    return LBM_OK;
}

}  // namespace lbm

#define LBM_INSTANTIATE_STEP(L, ST)                                                        \
    template int lbm::launch_step<lbm::L, ST>(const lbm::StepArgs&, int, int, int, int, cudaStream_t); \
    template int lbm::step_resources<lbm::L, ST>(int, int32_t*);
