// Batched domains: many independent lattices of different sizes advanced by
// one persistent launch per time step.
//
// Every block walks the tile list round-robin (item = blockIdx.x,
// blockIdx.x + gridDim.x, ...). A tile rebuilds the step arguments of its
// domain from the descriptor (a few cached loads) and runs exactly the
// per-node code of the single-domain step (bulk_node), so a batched domain
// evolves bit for bit like the same domain advanced alone.
// Blocks never wait on each other.
#include "dispatch.cuh"
#include "step_kernels.cuh"

namespace lbm {

struct BatchArgs {
    const lbm_domain_t* domains;
    const int4* tiles;
    int n_tiles;
    const uint8_t* kind;
    const uint32_t* nbr;
    const void* wall;
    const void* f_src;
    void* f_dst;
    uint32_t* seed;  // step counter of the stochastic rounding (16-bit storage)
    int parity;
};

template <class L, int ST>
__device__ __forceinline__ StepArgs domain_args(const BatchArgs& b, int d)
{
    const lbm_domain_t& D = b.domains[d];
    StepArgs a;
    a.nx = D.nx;
    a.ny = D.ny;
    a.nz = D.nz;
    a.pitch = D.pitch;
    a.qstride = D.qstride;
    a.wp = D.omega_plus;
    a.wm = D.omega_minus;
    a.fx = D.force[0];
    a.fy = D.force[1];
    a.fz = D.force[2];
    a.kind = b.kind + D.kind_offset;
    a.nbr = b.nbr + D.kind_offset;
    using T = typename Storage<ST>::T;
    using R = typename Storage<ST>::R;
    a.f_src = static_cast<const T*>(b.f_src) + D.offset;
    a.f_dst = static_cast<T*>(b.f_dst) + D.offset;
    a.wall_u = (b.wall != nullptr && D.wall_offset >= 0) ? static_cast<const R*>(b.wall) + D.wall_offset : nullptr;
    a.force_field = nullptr;
    a.seed = b.seed;
    a.parity = b.parity;
    // collision scalars per tile; force terms per node (no per-domain tables)
    a.guo_const = false;
    if constexpr (ST == LBM_F64)
        relax_scalars<L, double>(a.rd, D.omega_plus, D.omega_minus);
    else
        relax_scalars<L, float>(a.rf, D.omega_plus, D.omega_minus);
    return a;
}

template <class L, int ST>
__global__ void __launch_bounds__(256, 1) lbm_batch_kernel(const BatchArgs b)
{
    if (b.seed != nullptr && blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0)
        b.seed[b.parity ^ 1] = b.seed[b.parity] + 1u;
    for (int item = blockIdx.x; item < b.n_tiles; item += gridDim.x) {
        const int4 t = b.tiles[item];
        const StepArgs a = domain_args<L, ST>(b, t.x);
        const int x = t.y * blockDim.x + threadIdx.x;
        const int y = t.z * blockDim.y + threadIdx.y;
        bulk_node<L, ST, LBM_PULL>(a, x, y, t.w, ((int64_t)t.w * a.ny + y) * a.pitch + x, x < a.nx && y < a.ny);
    }
}

template <class L, int ST>
int batch_step(const lbm_batch_t& bt, const void* src, void* dst, cudaStream_t s)
{
    BatchArgs b;
    b.domains = bt.domains;
    b.tiles = reinterpret_cast<const int4*>(bt.tiles);
    b.n_tiles = bt.n_tiles;
    b.kind = bt.kind;
    b.nbr = bt.solid_nbr;
    b.wall = bt.wall_u;
    b.f_src = src;
    b.f_dst = dst;
    b.seed = (bt.storage == LBM_F16 || bt.storage == LBM_BF16) ? bt.round_seed : nullptr;
    b.parity = (uintptr_t)src > (uintptr_t)dst ? 1 : 0;
    lbm_batch_kernel<L, ST><<<bt.blocks, dim3(bt.tile_x, bt.tile_y), 0, s>>>(b);
    return launch_status();
}

template <class L, int ST>
int batch_occupancy(int tile_x, int tile_y, int32_t* out)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, lbm_batch_kernel<L, ST>, tile_x * tile_y, 0) != cudaSuccess)
        return LBM_ERR_LAUNCH;
    *out = n;
    return LBM_OK;
}

}  // namespace lbm

using namespace lbm;

extern "C" int lbm_batch_step(const lbm_batch_t* bt, const void* f_src, void* f_dst, lbm_stream_t stream)
{
    if (!bt || !f_src || !f_dst || f_src == f_dst || !bt->domains || !bt->kind || !bt->solid_nbr || bt->n_domains <= 0)
        return LBM_ERR_INVALID;
    if (bt->n_tiles < 0 || (bt->n_tiles > 0 && !bt->tiles)) return LBM_ERR_INVALID;
    if (bt->tile_x <= 0 || bt->tile_y <= 0 || bt->tile_x % 32 || bt->tile_x * bt->tile_y > 256 || bt->blocks <= 0)
        return LBM_ERR_INVALID;
    if ((bt->storage == LBM_F16 || bt->storage == LBM_BF16) && !bt->round_seed) return LBM_ERR_INVALID;
    LBM_DISPATCH(bt->lattice, bt->storage, batch_step, *bt, f_src, f_dst, (cudaStream_t)stream);
}

extern "C" int lbm_batch_occupancy(int32_t lattice, int32_t storage, int32_t tile_x, int32_t tile_y, int32_t* out)
{
    if (!out || tile_x <= 0 || tile_y <= 0 || tile_x * tile_y > 256) return LBM_ERR_INVALID;
    LBM_DISPATCH(lattice, storage, batch_occupancy, tile_x, tile_y, out);
}
