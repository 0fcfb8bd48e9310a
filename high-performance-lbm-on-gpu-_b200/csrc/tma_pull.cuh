// TMA-staged two-lattice pull for 16-bit storage (sm_100a).
//
// Each persistent block walks a list of tiles: TMA_ROWS consecutive rows
// (y) of one z plane, whole rows along x. For every direction i the tile's
// source rows -- the same rows shifted by -c_i in y and z, whole rows in x --
// are brought into shared memory by one cp.async.bulk.tensor load (4-D
// tensor map over x, y, z, direction; no multicast), so one tile needs Q
// loads and the warps never wait on global memory: while they update one
// tile, the loads of the next TMA_STAGES - 1 tiles of the block are in
// flight into the other stages. Completion is tracked by an mbarrier per
// stage (transaction bytes).
//
// Links along x read the staged row at x - c_x, wrapped periodically inside
// the row, so x shifts cost nothing. Each thread updates node pairs (x even,
// x + 1): two independent collisions, one cvt.rs per direction for both
// results (stochastic rounding, see sr_pair_hash), one 4-byte store.
//
// The tile's kind bytes are staged with it. A warp takes this path when
// each of its fluid nodes lies off the y and z faces of the box (so every
// staged source row exists); links from solid neighbours bounce back from
// the node's own slots (solid-neighbour mask), and solid and SPECIAL nodes
// are left alone. Any other warp -- fluid nodes on a periodic y or z face --
// updates its nodes one by one from global memory (bulk_node). Per node the
// arithmetic and the rounding are those of the one-node paths.
//
// Every wait on an mbarrier is bounded: if a stage has not arrived after
// a.wait_limit polls (lbm_launch_t.tma_wait_limit, default
// WAIT_LIMIT_DEFAULT), the block sets status[0] (the caller's status word),
// waits for the loads it still has in flight (bounded by the default limit,
// so that none is outstanding when the block exits) and returns.
#pragma once

#include <cuda.h>

#include "lbm_common.cuh"

namespace lbm {

// Tile shape and pipeline depth, from a sweep on B200 (256^3 duct, float16):
// 2-row tiles, 128 threads, 2 stages and 5 blocks per SM (200 KB of shared
// memory) measured 71 GLUPS; 4-row tiles or 256-512 threads with deeper
// pipelines and fewer blocks per SM 47-66 GLUPS.
constexpr int TMA_ROWS = 2;
constexpr int TMA_THREADS = 128;
constexpr int TMA_STAGES = 2;  // tiles in flight per block: TMA_STAGES - 1 ahead of the one computed
constexpr int TMA_BLOCKS_PER_SM = 5;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return done != 0u;
}

// Bounded wait (`limit` polls) for the phase `phase` of `bar` to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint32_t limit)
{
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z, int w)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];"
        ::"r"(smem_addr(dst)), "l"(map), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
        : "memory");
}

// Shared memory of one stage: the Q staged directions (TMA_ROWS x nx
// populations each), then the tile's kind bytes, padded to 128 bytes.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_addr(dst)), "l"(map), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Bulk tensor store of a shared-memory tile (x must be a multiple of 8 nodes
// for 16-bit data; every store here starts at x = 0 and y, z >= 0).
__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, const void* src, int x, int y, int z, int w)
{
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];"
                 ::"l"(map), "r"(smem_addr(src)), "r"(x), "r"(y), "r"(z), "r"(w)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// The committed stores have finished reading shared memory ...
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... and have completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Shared-memory writes of this thread become visible to the bulk-copy (async) proxy.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <class L>
__host__ __device__ constexpr uint32_t tma_pop_bytes(int nx)
{
    return (uint32_t)L::Q * TMA_ROWS * (uint32_t)nx * 2u;
}
template <class L>
__host__ __device__ constexpr uint32_t tma_stage_bytes(int nx)
{
    return (tma_pop_bytes<L>(nx) + TMA_ROWS * (uint32_t)nx + 127u) & ~127u;
}
// The odd AA half's output buffer (one tile of populations; a multiple of 128 bytes).
template <class L, int VAR>
__host__ __device__ constexpr uint32_t tma_out_bytes(int nx)
{
    return VAR == LBM_AA_ODD ? tma_pop_bytes<L>(nx) : 0u;
}
template <class L, int VAR>
__host__ __device__ constexpr uint32_t tma_smem_bytes(int nx)
{
    return TMA_STAGES * tma_stage_bytes<L>(nx) + tma_out_bytes<L, VAR>(nx) + 8u * TMA_STAGES;
}

// Halfway bounce-back on the staged path: each link i whose source x - c_i
// is solid (bit i of the node's solid-neighbour mask) takes f*_opp(i) of the
// node itself from global memory, plus the moving-wall term, in the
// collision's units (times 2^SCALE_LOG2; exact), as the one-node paths do.
template <class L, int ST>
__device__ __forceinline__ void bounce(const StepArgs& a, typename Storage<ST>::R (&f)[L::Q], int64_t nd, int x, int y, int z)
{
    using S = Storage<ST>;
    using R = typename S::R;
    const R* __restrict__ wall = static_cast<const R*>(a.wall_u);
    const unsigned short* fs = static_cast<const unsigned short*>(a.f_src);
    uint32_t m = a.nbr[nd] & ~1u;
    while (m) {
        const int i = __ffs(m) - 1;
        m &= m - 1u;
        R v = S::decode_lo(__ldg(fs + (int64_t)L::opp(i) * a.qstride + nd));
        R w = R(0);  // added even when zero, as the one-node paths do (-0 + 0 = +0)
        if (wall != nullptr) {
            const int sx = wrap(x - L::cx(i), a.nx), sy = wrap(y - L::cy(i), a.ny);
            const int sz = L::D == 3 ? wrap(z - L::cz(i), a.nz) : 0;
            w = wall_term<L, R>(i, wall, ((int64_t)sz * a.ny + sy) * a.pitch + sx, a.qstride);
            if (S::SCALE_LOG2) w = v_mul(w, R(1 << S::SCALE_LOG2));
        }
        v = v_add(v, w);
#pragma unroll
        for (int j = 1; j < L::Q; ++j)
            if (j == i) f[j] = v;
    }
}

// The streamed populations of pair (x0, x0 + 1) from a staged row set (the
// odd AA half and the pull: direction i's row at st_row + i * plane, staged
// from the source rows y - c_y, z - c_z; x - c_x read in the row, wrapped).
template <class L, int ST>
__device__ __forceinline__ void staged_gather(const typename Storage<ST>::T* st_row, int plane, int x0, int nx,
                                              typename Storage<ST>::R (&fa)[L::Q], typename Storage<ST>::R (&fb)[L::Q])
{
    using S = Storage<ST>;
    const int xm = x0 == 0 ? nx - 1 : x0 - 1;  // x0 - 1, wrapped
    const int xp = x0 + 2 == nx ? 0 : x0 + 2;  // x0 + 2, wrapped
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        const unsigned short* row = reinterpret_cast<const unsigned short*>(st_row + i * plane);
        if (L::cx(i) == 0) {
            const uint32_t w = *reinterpret_cast<const uint32_t*>(row + x0);
            fa[i] = S::decode_lo(w);
            fb[i] = S::decode_hi(w);
        } else if (L::cx(i) > 0) {  // sources x0 - 1, x0
            fa[i] = S::decode_lo(row[xm]);
            fb[i] = S::decode_lo(row[x0]);
        } else {  // sources x0 + 1, x0 + 2
            fa[i] = S::decode_lo(row[x0 + 1]);
            fb[i] = S::decode_lo(row[xp]);
        }
    }
}

// Odd AA half of an interior pair, outputs staged for bulk stores: out_row is
// direction 0's row of the tile's output buffer (direction i at out_row + i *
// plane), holding in destination order the values that the whole rows y + c_y,
// z + c_z of slot i receive: node x pushes f*_i to x + c_x (wrapped in the row).
template <class L, int ST>
__device__ __forceinline__ void tma_aa_odd_staged(const StepArgs& a, const typename Storage<ST>::T* st_row, int plane,
                                                  unsigned short* out_row, int x0, int y, int z,
                                                  const Relax<typename Storage<ST>::R>& rc, uint32_t t_seed)
{
    using S = Storage<ST>;
    using R = typename S::R;
    constexpr int Q = L::Q;
    const int nx = a.nx;
    R fa[Q], fb[Q];
    staged_gather<L, ST>(st_row, plane, x0, nx, fa, fb);
    collide_pair<L, S::SCALE_LOG2>(fa, fb, rc, R(a.fx), R(a.fy), R(a.fz));
    const uint32_t h = sr_pair_hash(sr_pair(nx, a.ny, x0, y, z), t_seed);
    const int xm = x0 == 0 ? nx - 1 : x0 - 1;
    const int xp = x0 + 2 == nx ? 0 : x0 + 2;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const uint32_t w = S::pack_sr(fa[i], fb[i], sr_word(h, i));  // (x0, x0 + 1) rounded
        unsigned short* o = out_row + i * plane;
        if (L::cx(i) == 0) {
            *reinterpret_cast<uint32_t*>(o + x0) = w;
        } else if (L::cx(i) > 0) {  // x0 -> x0 + 1, x0 + 1 -> x0 + 2
            o[x0 + 1] = (unsigned short)w;
            o[xp] = (unsigned short)(w >> 16);
        } else {  // x0 -> x0 - 1, x0 + 1 -> x0
            o[xm] = (unsigned short)w;
            o[x0] = (unsigned short)(w >> 16);
        }
    }
}

// One pair (x0, x0 + 1) of staged row r of an AA tile; st_row: direction 0's
// staged row (direction i at st_row + i * plane), kind_row: the row's kinds.
template <class L, int ST, int VAR>
__device__ __forceinline__ void tma_aa_pair(const StepArgs& a, const typename Storage<ST>::T* st_row, int plane,
                                            const unsigned char* kind_row, int x0, int y, int z,
                                            const Relax<typename Storage<ST>::R>& rc, uint32_t t_seed)
{
    using S = Storage<ST>;
    using T = typename S::T;
    using R = typename S::R;
    constexpr int Q = L::Q;
    constexpr unsigned FULL = 0xffffffffu;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int64_t qs = a.qstride;
    const int64_t nd0 = ((int64_t)z * ny + y) * a.pitch + x0;
    const uint32_t k2 = *reinterpret_cast<const unsigned short*>(kind_row + x0);
    const R Fx = R(a.fx), Fy = R(a.fy), Fz = R(a.fz);
    R fa[Q], fb[Q];
    if constexpr (VAR == LBM_AA_EVEN) {
        const bool skip_a = (k2 & (KIND_SOLID | KIND_SPECIAL)) != 0u;
        const bool skip_b = ((k2 >> 8) & (KIND_SOLID | KIND_SPECIAL)) != 0u;
        if (y >= ny || (skip_a && skip_b)) return;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const uint32_t w = *reinterpret_cast<const uint32_t*>(st_row + i * plane + x0);
            fa[i] = S::decode_lo(w);
            fb[i] = S::decode_hi(w);
        }
        collide_pair<L, S::SCALE_LOG2>(fa, fb, rc, Fx, Fy, Fz);
        const uint32_t h = sr_pair_hash(sr_pair(nx, ny, x0, y, z), t_seed);
        T* fd = static_cast<T*>(a.f_dst) + nd0;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const uint32_t w = S::pack_sr(fa[i], fb[i], sr_word(h, i));
            T* d = fd + L::opp(i) * qs;
            if (!skip_a && !skip_b) {
                *reinterpret_cast<uint32_t*>(d) = w;
            } else {
                if (!skip_a) *reinterpret_cast<unsigned short*>(d) = (unsigned short)w;
                if (!skip_b) *reinterpret_cast<unsigned short*>(d + 1) = (unsigned short)(w >> 16);
            }
        }
    } else {
        const bool staged = y >= 1 && y <= ny - 2 && (L::D == 2 || (z >= 1 && z <= nz - 2));
        const bool ok = staged && (k2 & ~0x0808u) == 0u;  // both nodes interior (x faces allowed)
        if (!__all_sync(FULL, ok)) {
            for (int h = 0; h < 2; ++h) bulk_node<L, ST, LBM_AA_ODD>(a, x0 + h, y, z, nd0 + h, y < ny);
            return;
        }
        const int lane = threadIdx.x & 31;
        const int xm = x0 == 0 ? nx - 1 : x0 - 1;  // x0 - 1, wrapped
        const int xp = x0 + 2 == nx ? 0 : x0 + 2;  // x0 + 2, wrapped
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const unsigned short* row = reinterpret_cast<const unsigned short*>(st_row + i * plane);
            if (L::cx(i) == 0) {
                const uint32_t w = *reinterpret_cast<const uint32_t*>(row + x0);
                fa[i] = S::decode_lo(w);
                fb[i] = S::decode_hi(w);
            } else if (L::cx(i) > 0) {  // sources x0 - 1, x0
                fa[i] = S::decode_lo(row[xm]);
                fb[i] = S::decode_lo(row[x0]);
            } else {  // sources x0 + 1, x0 + 2
                fa[i] = S::decode_lo(row[x0 + 1]);
                fb[i] = S::decode_lo(row[xp]);
            }
        }
        collide_pair<L, S::SCALE_LOG2>(fa, fb, rc, Fx, Fy, Fz);
        const uint32_t h = sr_pair_hash(sr_pair(nx, ny, x0, y, z), t_seed);
        // the warp's 64 nodes: [x_base, x_base + 64); the nodes beyond, wrapped
        const int x_base = x0 - 2 * lane;
        const int x_lo = x_base == 0 ? nx - 1 : x_base - 1;
        const int x_hi = x_base + 64 == nx ? 0 : x_base + 64;
        T* f = static_cast<T*>(a.f_dst);
        const int64_t pz = (int64_t)a.pitch * ny;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const uint32_t w = S::pack_sr(fa[i], fb[i], sr_word(h, i));  // (x0, x0 + 1) rounded
            T* dst_row = f + i * qs + ((int64_t)z * ny + y) * a.pitch + (L::cy(i) * a.pitch + L::cz(i) * pz);
            if (L::cx(i) == 0) {
                *reinterpret_cast<uint32_t*>(dst_row + x0) = w;
            } else if (L::cx(i) > 0) {  // pair (x0, x0 + 1) <- (lane - 1's odd node, own even node)
                const uint32_t pw = __shfl_up_sync(FULL, w, 1);
                if (lane == 0)
                    *reinterpret_cast<unsigned short*>(dst_row + x0 + 1) = (unsigned short)(w & 0xffffu);
                else
                    *reinterpret_cast<uint32_t*>(dst_row + x0) = __byte_perm(pw, w, 0x5432);
                if (lane == 31) *reinterpret_cast<unsigned short*>(dst_row + x_hi) = (unsigned short)(w >> 16);
            } else {  // pair (x0, x0 + 1) <- (own odd node, lane + 1's even node)
                const uint32_t nw = __shfl_down_sync(FULL, w, 1);
                if (lane == 31)
                    *reinterpret_cast<unsigned short*>(dst_row + x0) = (unsigned short)(w >> 16);
                else
                    *reinterpret_cast<uint32_t*>(dst_row + x0) = __byte_perm(w, nw, 0x5432);
                if (lane == 0) *reinterpret_cast<unsigned short*>(dst_row + x_lo) = (unsigned short)(w & 0xffffu);
            }
        }
    }
}

// The staged step for one variant. PULL as described above. AA (in place,
// one lattice; the caller requires nx >= 64, so a warp's 32 pairs are 64
// consecutive nodes of one row):
//   * AA_EVEN: the tile's own rows of slot i are staged; each pair is
//     node-local (slot i in, slot opp(i) out), solid and SPECIAL nodes are
//     skipped with 2-byte stores.
//   * AA_ODD: rows y - c_y, z - c_z of slot opp(i) are staged; a warp of
//     interior nodes (kinds 0 and EDGE, rows off the y and z faces) computes
//     its pairs and pushes slot i to x + c_i: destination pairs straddle
//     the source pairs along x, so each lane rounds its own two results and a
//     shuffle hands the crossing half to the neighbouring lane; the half that
//     leaves the warp's 64 nodes is stored alone by lane 0 or 31 (x wrapped
//     in the row), and every slot is written once. Other warps update their
//     nodes one by one (bulk_node).
// In place is safe with loads in flight: slot (j, row) is read and written
// only by the tile that owns its source node (the rows of a tile are whole
// and x wraps inside them).
template <class L, int ST, int VAR>
__device__ __forceinline__ void tma_step(const CUtensorMap& map, const CUtensorMap& kmap, const StepArgs& a,
                                         uint32_t* status)
{
    using S = Storage<ST>;
    using T = typename S::T;
    using R = typename S::R;
    constexpr int Q = L::Q;
    constexpr int H = TMA_ROWS;
    static_assert(sizeof(T) == 2, "16-bit storage");
    extern __shared__ __align__(128) unsigned char smem[];

    const int nx = a.nx, ny = a.ny, nz = a.nz;  // nx: a power of two in [32, 256]
    const int tiles_y = (ny + H - 1) / H;
    const int n_tiles = nz * tiles_y;
    const uint32_t pop_bytes = tma_pop_bytes<L>(nx);
    const uint32_t tx_bytes = pop_bytes + H * nx;
    const uint32_t stage_bytes = tma_stage_bytes<L>(nx);
    const int plane = H * nx;  // populations per staged direction
    const int log_half = __ffs(nx) - 2;  // log2(nx / 2)
    // the odd AA half stages its outputs for bulk stores in a buffer after the stages
    unsigned short* out = reinterpret_cast<unsigned short*>(smem + TMA_STAGES * stage_bytes);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + TMA_STAGES * stage_bytes + tma_out_bytes<L, VAR>(nx));
    const int tid = threadIdx.x;

    advance_seed(a);
    if (tid == 0) {
        for (int k = 0; k < TMA_STAGES; ++k) mbar_init(&bar[k], 1);
        mbar_init_fence();
    }
    __syncthreads();

    auto issue = [&](int z, int y0, int s) {
        unsigned char* dst = smem + s * stage_bytes;
        mbar_expect_tx(&bar[s], tx_bytes);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            if (VAR == LBM_AA_EVEN)
                tma_load_4d(dst + (size_t)i * plane * 2, &map, &bar[s], 0, y0, z, i);
            else
                tma_load_4d(dst + (size_t)i * plane * 2, &map, &bar[s], 0, y0 - L::cy(i), z - L::cz(i),
                            VAR == LBM_PULL ? i : L::opp(i));
        }
        tma_load_3d(dst + pop_bytes, &kmap, &bar[s], 0, y0, z);
    };

    const Relax<R>& rc = a.template relax<R>();
    const R Fx = R(a.fx), Fy = R(a.fy), Fz = R(a.fz);
    const uint32_t t_seed = a.seed[a.parity];
    const int64_t qs = a.qstride;
    T* fd_base = static_cast<T*>(a.f_dst);

    // tiles blockIdx.x, blockIdx.x + gridDim.x, ... as (z, row block); the
    // stride is split once so that no tile needs a division. (iz, iy) runs
    // TMA_STAGES - 1 tiles ahead of (tz, ty): the next tile to issue.
    const int dz = gridDim.x / tiles_y, dy = gridDim.x - dz * tiles_y;
    int tz = blockIdx.x / tiles_y, ty = blockIdx.x - tz * tiles_y;
    int iz = tz, iy = ty, itile = blockIdx.x;
    uint32_t phases = 0u;  // bit k: parity of the next completion of stage k
    uint32_t issued = 0u;  // bit k: stage k has loads in flight
    for (int k = 0; k < TMA_STAGES - 1 && itile < n_tiles; ++k) {
        if (tid == 0) issue(iz, iy * H, k);
        issued |= 1u << k;
        itile += gridDim.x;
        iy += dy;
        iz += dz;
        if (iy >= tiles_y) {
            iy -= tiles_y;
            ++iz;
        }
    }
    int s = 0;
    bool failed = false;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        if (itile < n_tiles) {
            const int si = s == 0 ? TMA_STAGES - 1 : s - 1;  // consumed in the previous iteration
            if (tid == 0) issue(iz, iy * H, si);
            issued |= 1u << si;
            itile += gridDim.x;
            iy += dy;
            iz += dz;
            if (iy >= tiles_y) {
                iy -= tiles_y;
                ++iz;
            }
        }
        const int z = tz, y0 = ty * H;
        ty += dy;
        tz += dz;
        if (ty >= tiles_y) {
            ty -= tiles_y;
            ++tz;
        }
        const bool arrived = mbar_wait(&bar[s], (phases >> s) & 1u, a.wait_limit);
        if (__syncthreads_or(!arrived)) {
            failed = true;
            break;
        }
        phases ^= 1u << s;
        issued &= ~(1u << s);
        const T* st = reinterpret_cast<const T*>(smem + s * stage_bytes);
        const unsigned char* kinds = smem + s * stage_bytes + pop_bytes;
        bool staged_out = false;
        if constexpr (VAR == LBM_AA_ODD) {
            // A tile of interior nodes only (kinds 0 and EDGE, rows off the y and z faces):
            // outputs into the buffer in destination order, then one bulk store per direction
            // of the whole rows y0 + c_y, z + c_z of slot i (every slot of them comes from this
            // tile: x wraps inside the row, and no push meets a wall).
            bool ok = true;
            for (int p = tid; p < plane / 2; p += TMA_THREADS) {
                const int r = p >> log_half;
                const int x0 = 2 * (p - (r << log_half));
                const int y = y0 + r;
                const uint32_t k2 = *reinterpret_cast<const unsigned short*>(kinds + r * nx + x0);
                ok = ok && y >= 1 && y <= ny - 2 && (L::D == 2 || (z >= 1 && z <= nz - 2)) && (k2 & ~0x0808u) == 0u;
            }
            if (__syncthreads_and(ok)) {
                if (tid == 0) bulk_wait_read();  // the previous tile's stores have read the buffer
                __syncthreads();
#pragma unroll 1
                for (int p = tid; p < plane / 2; p += TMA_THREADS) {
                    const int r = p >> log_half;
                    const int x0 = 2 * (p - (r << log_half));
                    tma_aa_odd_staged<L, ST>(a, st + r * nx, plane, out + r * nx, x0, y0 + r, z, rc, t_seed);
                }
                fence_proxy_async();
                __syncthreads();
                if (tid == 0) {
#pragma unroll
                    for (int i = 0; i < Q; ++i) tma_store_4d(&map, out + i * plane, 0, y0 + L::cy(i), z + L::cz(i), i);
                    bulk_commit();
                }
                staged_out = true;
            }
        }
#pragma unroll 1
        for (int p = staged_out ? plane / 2 : tid; p < plane / 2; p += TMA_THREADS) {
            const int r = p >> log_half;
            const int x0 = 2 * (p - (r << log_half));
            const int y = y0 + r;
            if constexpr (VAR != LBM_PULL) {
                tma_aa_pair<L, ST, VAR>(a, st + r * nx, plane, kinds + r * nx, x0, y, z, rc, t_seed);
                continue;
            }
            // A fluid node takes the staged path when its source rows exist
            // (y, z inside the box faces); solid and SPECIAL nodes are left
            // alone (the boundary warps update the latter).
            const uint32_t k2 = *reinterpret_cast<const unsigned short*>(kinds + r * nx + x0);
            const bool skip_a = (k2 & (KIND_SOLID | KIND_SPECIAL)) != 0u;
            const bool skip_b = ((k2 >> 8) & (KIND_SOLID | KIND_SPECIAL)) != 0u;
            const bool staged = y >= 1 && y <= ny - 2 && (L::D == 2 || (z >= 1 && z <= nz - 2));
            const bool ok = y < ny && (staged || (skip_a && skip_b));
            const int64_t nd0 = ((int64_t)z * ny + y) * a.pitch + x0;
            if (!__all_sync(0xffffffffu, ok)) {
                for (int h = 0; h < 2; ++h) bulk_node<L, ST, LBM_PULL>(a, x0 + h, y, z, nd0 + h, y < ny);
            } else if (!(skip_a && skip_b)) {
                const int xm = x0 == 0 ? nx - 1 : x0 - 1;  // x0 - 1, wrapped
                const int xp = x0 + 2 == nx ? 0 : x0 + 2;  // x0 + 2, wrapped
                R fa[Q], fb[Q];
#pragma unroll
                for (int i = 0; i < Q; ++i) {
                    const unsigned short* row = reinterpret_cast<const unsigned short*>(st + i * plane + r * nx);
                    if (L::cx(i) == 0) {
                        const uint32_t w = *reinterpret_cast<const uint32_t*>(row + x0);
                        fa[i] = S::decode_lo(w);
                        fb[i] = S::decode_hi(w);
                    } else if (L::cx(i) > 0) {  // sources x0 - 1, x0
                        fa[i] = S::decode_lo(row[xm]);
                        fb[i] = S::decode_lo(row[x0]);
                    } else {  // sources x0 + 1, x0 + 2
                        fa[i] = S::decode_lo(row[x0 + 1]);
                        fb[i] = S::decode_lo(row[xp]);
                    }
                }
                // next to a wall: links from solid nodes bounce back
                if ((k2 & KIND_NEAR) && !skip_a) bounce<L, ST>(a, fa, nd0, x0, y, z);
                if (((k2 >> 8) & KIND_NEAR) && !skip_b) bounce<L, ST>(a, fb, nd0 + 1, x0 + 1, y, z);
                collide_pair<L, S::SCALE_LOG2>(fa, fb, rc, Fx, Fy, Fz);
                const uint32_t h = sr_pair_hash(sr_pair(nx, ny, x0, y, z), t_seed);
                T* fd = fd_base + nd0;
                if (!skip_a && !skip_b) {
#pragma unroll
                    for (int i = 0; i < Q; ++i)
                        *reinterpret_cast<uint32_t*>(fd + i * qs) = S::pack_sr(fa[i], fb[i], sr_word(h, i));
                } else {
#pragma unroll
                    for (int i = 0; i < Q; ++i) {
                        const uint32_t w = S::pack_sr(fa[i], fb[i], sr_word(h, i));
                        unsigned short* d = reinterpret_cast<unsigned short*>(fd + i * qs);
                        if (!skip_a) d[0] = (unsigned short)w;
                        if (!skip_b) d[1] = (unsigned short)(w >> 16);
                    }
                }
            }
        }
        __syncthreads();  // the stage is read; the next issue may overwrite it
        s = s + 1 == TMA_STAGES ? 0 : s + 1;
    }
    if (failed) {
        if (tid == 0) atomicOr(status, 1u);
        // wait (bounded) for the loads still in flight into this block's stages
        for (int k = 0; k < TMA_STAGES; ++k)
            if ((issued >> k) & 1u) mbar_wait(&bar[k], (phases >> k) & 1u, WAIT_LIMIT_DEFAULT);
    }
    // no bulk store may still read shared memory when the block exits
    if constexpr (VAR == LBM_AA_ODD) {
        if (tid == 0) bulk_wait_all();
    }
}

template <class L, int ST>
__global__ void __launch_bounds__(TMA_THREADS, TMA_BLOCKS_PER_SM) lbm_tma_pull_kernel(const __grid_constant__ CUtensorMap map,
                                                                      const __grid_constant__ CUtensorMap kmap,
                                                                      const StepArgs a, uint32_t* status)
{
    tma_step<L, ST, LBM_PULL>(map, kmap, a, status);
}

// The odd AA half holds a third buffer of shared memory (its staged outputs),
// so three blocks fit on an SM, not five: its register bound follows.
template <int VAR>
constexpr int tma_min_blocks() { return VAR == LBM_AA_ODD ? 3 : TMA_BLOCKS_PER_SM; }

template <class L, int ST, int VAR>
__global__ void __launch_bounds__(TMA_THREADS, tma_min_blocks<VAR>()) lbm_tma_aa_kernel(const __grid_constant__ CUtensorMap map,
                                                                    const __grid_constant__ CUtensorMap kmap,
                                                                    const StepArgs a, uint32_t* status)
{
    tma_step<L, ST, VAR>(map, kmap, a, status);
}

// Driver entry point for tensor-map encoding (no link-time dependency on
// the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled_fn()
{
    static EncodeTiledFn fn = []() -> EncodeTiledFn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

template <class L, int ST, int VAR>
constexpr auto tma_kernel()
{
    if constexpr (VAR == LBM_PULL)
        return lbm_tma_pull_kernel<L, ST>;
    else
        return lbm_tma_aa_kernel<L, ST, VAR>;
}

// Launch the TMA-staged step (pull, or one AA half in place) if the grid
// qualifies; returns false (nothing launched) when it does not, so the
// caller can take another kernel.
template <class L, int ST, int VAR>
bool launch_tma(const StepArgs& a, cudaStream_t stream, int* status_out)
{
    *status_out = LBM_OK;
    // Whole rows of a power-of-two width in one box; rows of 16-byte
    // multiples. nx >= 32: a tile then holds at least 32 pairs, so every
    // warp that reaches the warp-wide votes is full, and each staged
    // direction (2 rows x nx x 2 bytes) is a multiple of 128 bytes, the
    // alignment of a TMA destination in shared memory. AA: nx >= 64, a
    // warp's 32 pairs within one row.
    const int nx_min = VAR == LBM_PULL ? 32 : 64;
    if (a.nx < nx_min || a.nx > 256 || (a.nx & (a.nx - 1)) != 0 || a.pitch % 16 != 0) return false;
    if (reinterpret_cast<uintptr_t>(a.kind) % 16 != 0) return false;
    if (a.force_field != nullptr || !a.guo_const || a.seed == nullptr) return false;
    if (reinterpret_cast<uintptr_t>(a.f_src) % 16 != 0 || reinterpret_cast<uintptr_t>(a.f_dst) % 4 != 0) return false;
    EncodeTiledFn encode = encode_tiled_fn();
    if (encode == nullptr) return false;
    CUtensorMap map;
    const cuuint64_t dims[4] = {(cuuint64_t)a.nx, (cuuint64_t)a.ny, (cuuint64_t)a.nz, (cuuint64_t)L::Q};
    const cuuint64_t strides[3] = {(cuuint64_t)a.pitch * 2, (cuuint64_t)a.pitch * a.ny * 2, (cuuint64_t)a.qstride * 2};
    const cuuint32_t box[4] = {(cuuint32_t)a.nx, (cuuint32_t)TMA_ROWS, 1, 1};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    if (encode(&map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, const_cast<void*>(a.f_src), dims, strides, box, elem,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    CUtensorMap kmap;  // the kind bytes of the same rows
    const cuuint64_t kdims[3] = {(cuuint64_t)a.nx, (cuuint64_t)a.ny, (cuuint64_t)a.nz};
    const cuuint64_t kstrides[2] = {(cuuint64_t)a.pitch, (cuuint64_t)a.pitch * a.ny};
    const cuuint32_t kbox[3] = {(cuuint32_t)a.nx, (cuuint32_t)TMA_ROWS, 1};
    if (encode(&kmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t*>(a.kind), kdims, kstrides, kbox, elem,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    const size_t smem = tma_smem_bytes<L, VAR>(a.nx);
    int device = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) {
        cudaGetLastError();
        return false;
    }
    // per device context: the shared-memory opt-in of this kernel (a new
    // context after cudaDeviceReset needs it again)
    static unsigned long long configured[64] = {};
    const unsigned long long ctx = current_context_id();
    if (ctx == 0 || configured[device] != ctx) {
        if (cudaFuncSetAttribute(tma_kernel<L, ST, VAR>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tma_smem_bytes<L, VAR>(256)) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        configured[device] = ctx;
    }
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tma_kernel<L, ST, VAR>(), TMA_THREADS, smem) !=
            cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return false;
    }
    const int64_t tiles = (int64_t)a.nz * ((a.ny + TMA_ROWS - 1) / TMA_ROWS);
    if (tiles > 0x7fffffff) return false;
    const int64_t grid = tiles < (int64_t)sms * per_sm ? tiles : (int64_t)sms * per_sm;
    tma_kernel<L, ST, VAR>()<<<(unsigned)grid, TMA_THREADS, smem, stream>>>(map, kmap, a, a.seed + 2);
    *status_out = cudaPeekAtLastError() == cudaSuccess ? LBM_OK : LBM_ERR_LAUNCH;
    return true;
}

}  // namespace lbm
