// extern "C" entry points of the step (include/lbm_b200.h).
#include "dispatch.cuh"

using namespace lbm;

static thread_local const char* g_last_error = "no error";

static int record(int status)
{
    if (status == LBM_ERR_LAUNCH) g_last_error = cudaGetErrorString(cudaGetLastError());
    return status;
}

namespace lbm {

bool grid_valid(const lbm_grid_t* g)
{
    if (g == nullptr) return false;
    if (g->lattice != LBM_D2Q9 && g->lattice != LBM_D3Q19) return false;
    if (g->storage < LBM_F32 || g->storage > LBM_BF16) return false;
    if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || g->pitch < g->nx) return false;
    if (g->lattice == LBM_D2Q9 && g->nz != 1) return false;
    return g->qstride >= (int64_t)g->pitch * g->ny * g->nz;
}

bool special_valid(const lbm_special_t* sp, bool aa)
{
    if (sp == nullptr) return true;
    if (sp->n_special < 0 || sp->n_rules < 0 || sp->n_terms < 0 || sp->n_local < 0 || sp->n_export < 0) return false;
    if (sp->n_special == 0) return true;
    if (!sp->node || !sp->rule_mask || !sp->rule_first || !sp->force_slot) return false;
    if (sp->n_rules > 0) {
        if (!sp->term_start || !sp->rule_const || !sp->term_coeff) return false;
        if (aa ? !sp->term_export : (!sp->term_dir || !sp->term_node)) return false;
        if (aa && (!sp->export_in || sp->n_export <= 0)) return false;
        if (sp->ut_start) {  // dense form
            if (aa ? !sp->ut_export : !sp->ut_slot) return false;
            if (!sp->rule_row || !sp->rule_dense || reinterpret_cast<uintptr_t>(sp->rule_dense) % 16 != 0) return false;
        }
    }
    if (aa && sp->n_export > 0 && (!sp->export_mask || !sp->export_first || !sp->export_out)) return false;
    if (sp->n_local > 0 && !sp->local_force) return false;
    return true;
}

// Partial slots of a checked step: the bulk grid's blocks, then (split) the
// boundary launch's or (fused) the extra planes'.
static int64_t health_partials(const lbm_grid_t* g, const lbm_special_t* sp, int tx, int ty, int mode)
{
    const int64_t gx = (g->nx + tx - 1) / tx, gy = (g->ny + ty - 1) / ty;
    const int64_t ns = sp ? sp->n_special : 0;
    if (mode == LBM_LAUNCH_FUSED) {
        const int64_t per_plane = gx * gy * tx * ty;
        const int64_t extra = ns > 0 ? (ns + per_plane - 1) / per_plane : 0;
        return gx * gy * (g->nz + extra);
    }
    return gx * gy * g->nz + (ns + BOUNDARY_THREADS - 1) / BOUNDARY_THREADS;
}

int make_args(StepArgs& a, const lbm_grid_t* g, const lbm_physics_t* p, const lbm_special_t* sp,
                     const lbm_launch_t* launch, const uint8_t* kind, const void* src, void* dst, int& tx, int& ty,
                     int& mode)
{
    tx = launch ? launch->tile_x : 32;
    ty = launch ? launch->tile_y : 4;
    mode = launch ? launch->mode : LBM_LAUNCH_FUSED;
    if (tx <= 0 || ty <= 0 || tx % 32 != 0 || tx * ty > 256) return LBM_ERR_INVALID;
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
    a.f_src = src;
    a.f_dst = dst;
    a.wall_u = p->wall_u;
    a.force_field = p->force_field;
    a.nbr = p->solid_nbr;
    if (!a.nbr) return LBM_ERR_INVALID;
    if (p->collision != LBM_COLLIDE_TRT && p->collision != LBM_COLLIDE_REGULARIZED &&
        p->collision != LBM_COLLIDE_CUMULANT)
        return LBM_ERR_INVALID;
    if (p->collision == LBM_COLLIDE_CUMULANT && g->lattice != LBM_D2Q9) return LBM_ERR_UNSUPPORTED;
    a.collision = p->collision;
    // 16-bit storage rounds stochastically and needs the step counter
    const bool half = g->storage == LBM_F16 || g->storage == LBM_BF16;
    if (half && !p->round_seed) return LBM_ERR_INVALID;
    a.seed = half ? p->round_seed : nullptr;
    a.parity = 0;
    a.health_words = nullptr;
    a.health_partial = nullptr;
    a.readout_rho = nullptr;
    a.readout_u = nullptr;
    a.health_slot0 = 0;
    a.wait_limit = WAIT_LIMIT_DEFAULT;
    if (launch && launch->tma_wait_limit) a.wait_limit = launch->tma_wait_limit == LBM_TMA_WAIT_NONE ? 0u : launch->tma_wait_limit;
    if (sp)
        a.sp = *sp;
    else
        memset(&a.sp, 0, sizeof(a.sp));
    if (launch && launch->health) {
        const lbm_health_t* h = launch->health;
        if (!h->words || !h->partial || h->n_partial != health_partials(g, sp, tx, ty, mode)) return LBM_ERR_INVALID;
        a.health_words = h->words;
        a.health_partial = h->partial;
        if ((h->rho == nullptr) != (h->u == nullptr)) return LBM_ERR_INVALID;
        a.readout_rho = h->rho;
        a.readout_u = h->u;
    }
    // collision constants, computed once per launch
    a.guo_const = true;
    if (g->lattice == LBM_D2Q9) {
        relax_constants<D2Q9, float>(a.rf, a.wp, a.wm, a.fx, a.fy, a.fz);
        relax_constants<D2Q9, double>(a.rd, a.wp, a.wm, a.fx, a.fy, a.fz);
    } else {
        relax_constants<D3Q19, float>(a.rf, a.wp, a.wm, a.fx, a.fy, a.fz);
        relax_constants<D3Q19, double>(a.rd, a.wp, a.wm, a.fx, a.fy, a.fz);
    }
    return LBM_OK;
}

}  // namespace lbm

template <class L, int ST>
static int step_dispatch(const StepArgs& a, int variant, int mode, int tx, int ty, cudaStream_t s)
{
    return launch_step<L, ST>(a, variant, mode, tx, ty, s);
}

extern "C" int lbm_step_pull(const lbm_grid_t* g, const lbm_physics_t* p, const lbm_special_t* sp,
                             const lbm_launch_t* launch, const uint8_t* kind, const void* f_src, void* f_dst,
                             lbm_stream_t stream)
{
    if (!grid_valid(g) || !p || !kind || !f_src || !f_dst || f_src == f_dst || !special_valid(sp, false))
        return LBM_ERR_INVALID;
    StepArgs a;
    int tx = 0, ty = 0, mode = 0;
    int st = make_args(a, g, p, sp, launch, kind, f_src, f_dst, tx, ty, mode);
    if (st != LBM_OK) return st;
    a.parity = (uintptr_t)f_src > (uintptr_t)f_dst ? 1 : 0;
    const int lattice = g->lattice, storage = g->storage;
    auto run = [&]() -> int { LBM_DISPATCH(lattice, storage, step_dispatch, a, LBM_PULL, mode, tx, ty, (cudaStream_t)stream); };
    return record(run());
}

extern "C" int lbm_step_aa(const lbm_grid_t* g, const lbm_physics_t* p, const lbm_special_t* sp,
                           const lbm_launch_t* launch, const uint8_t* kind, void* f, int32_t parity,
                           lbm_stream_t stream)
{
    if (!grid_valid(g) || !p || !kind || !f || !special_valid(sp, true)) return LBM_ERR_INVALID;
    if (parity != LBM_AA_EVEN && parity != LBM_AA_ODD) return LBM_ERR_INVALID;
    StepArgs a;
    int tx = 0, ty = 0, mode = 0;
    int st = make_args(a, g, p, sp, launch, kind, f, f, tx, ty, mode);
    if (st != LBM_OK) return st;
    a.parity = parity == LBM_AA_ODD ? 1 : 0;
    const int lattice = g->lattice, storage = g->storage;
    auto run = [&]() -> int { LBM_DISPATCH(lattice, storage, step_dispatch, a, parity, mode, tx, ty, (cudaStream_t)stream); };
    return record(run());
}

extern "C" int64_t lbm_health_partials(const lbm_grid_t* g, const lbm_special_t* sp, const lbm_launch_t* launch)
{
    if (!grid_valid(g) || !launch || (sp && sp->n_special < 0)) return LBM_ERR_INVALID;
    const int tx = launch->tile_x, ty = launch->tile_y, mode = launch->mode;
    if (tx <= 0 || ty <= 0 || tx % 32 != 0 || tx * ty > 256) return LBM_ERR_INVALID;
    if (mode < LBM_LAUNCH_FUSED || mode > LBM_LAUNCH_BOUNDARY) return LBM_ERR_INVALID;
    return health_partials(g, sp, tx, ty, mode);
}

template <class L, int ST>
static int resources_dispatch(int which, int32_t* out4)
{
    return step_resources<L, ST>(which, out4);
}

extern "C" int lbm_kernel_resources(int32_t lattice, int32_t storage, int32_t which, int32_t* out4)
{
    if (!out4) return LBM_ERR_INVALID;
    auto run = [&]() -> int { LBM_DISPATCH(lattice, storage, resources_dispatch, which, out4); };
    return record(run());
}

extern "C" const char* lbm_last_cuda_error(void) { return g_last_error; }

extern "C" int32_t lbm_abi_version(void) { return 9; }
