/*
 * lbm_b200.h -- C ABI of liblbm_b200.so, the B200 (sm_100a) lattice Boltzmann step.
 *
 * Plain pointers and sizes only. Every device pointer is memory the caller
 * owns (the Python host side allocates it with PyTorch); the library keeps no
 * device allocations of its own. Every call is asynchronous on the given CUDA
 * stream and returns LBM_OK or an error code (never exits, never traps).
 *
 * Population layout: structure of arrays f[q][z][y][x_pitched]. A direction
 * plane holds qstride = pitch * ny * nz elements; x runs fastest with a row
 * pitch >= nx (padding columns are never read or written by the step). The
 * stored value is the shifted population f~ = f - w_q in the storage format.
 * In 2D nz = 1.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* lbm_stream_t; /* a cudaStream_t; NULL = legacy default stream */

/* ---- status codes ---------------------------------------------------- */
enum {
    LBM_OK = 0,
    LBM_ERR_INVALID = -1,      /* bad argument (null pointer, size, enum)   */
    LBM_ERR_UNSUPPORTED = -2,  /* combination not built into this library   */
    LBM_ERR_LAUNCH = -3        /* kernel launch failed; see lbm_last_cuda_error */
};

/* ---- enums ------------------------------------------------------------ */
enum { LBM_D2Q9 = 0, LBM_D3Q19 = 1 };
enum { LBM_F32 = 0, LBM_F64 = 1, LBM_F16 = 2, LBM_BF16 = 3 };
enum { LBM_PULL = 0, LBM_AA_EVEN = 1, LBM_AA_ODD = 2 };
/* Where a stored state keeps f*_k(y) (reference src/lbm/link_rules.py:16-25). */
enum { LBM_LAYOUT_PULL = 0, LBM_LAYOUT_AA_ODD = 1, LBM_LAYOUT_AA_EVEN = 2 };
/* Node kind bits (one byte per node). */
enum { LBM_KIND_SOLID = 1, LBM_KIND_SPECIAL = 2, LBM_KIND_NEAR = 4 };

/* ---- descriptors ------------------------------------------------------ */
typedef struct lbm_grid {
    int32_t lattice;   /* LBM_D2Q9 or LBM_D3Q19 */
    int32_t storage;   /* LBM_F32, LBM_F64, LBM_F16, LBM_BF16 */
    int32_t nx, ny, nz;
    int32_t pitch;     /* row pitch in nodes, >= nx */
    int64_t qstride;   /* pitch * ny * nz */
} lbm_grid_t;

/* Collision constants and wall data. "real" arrays use the compute type:
 * double for LBM_F64 storage, float otherwise. */
typedef struct lbm_physics {
    double omega_plus;     /* 1/tau */
    double omega_minus;    /* TRT antisymmetric rate (== omega_plus for BGK) */
    double force[3];       /* uniform body-force density */
    const void* wall_u;    /* real[d][qstride] wall velocity at solid nodes, or NULL (all walls at rest) */
    const void* force_field; /* real[d][qstride] per-node body force added to force[], or NULL */
} lbm_physics_t;

/* Nodes updated by the boundary warps, and the link rules they apply.
 * A rule sets the streamed population f_j(x) of a link from a resting solid
 * node x - c_j:  f_j(x) = const[r] + sum_t coeff[t] * f*_{dir[t]}(node[t]).
 * Rules of one node are consecutive and sorted by direction. */
typedef struct lbm_special {
    int32_t n_special;
    const int64_t* node;          /* pitched node index of each special node */
    const uint32_t* rule_mask;    /* bit j: f_j of this node comes from a rule */
    const int32_t* rule_first;    /* index of the node's first rule */
    const int32_t* force_slot;    /* column of local_force, or -1 */
    const uint32_t* export_mask;  /* AA: bit k: this node exports f*_k(node) */
    const int32_t* export_first;  /* AA: export index of the node's first export */
    int32_t n_rules;
    int32_t n_terms;
    const int32_t* term_start;    /* n_rules + 1 offsets into the term arrays */
    const void* rule_const;       /* real[n_rules] */
    const int32_t* term_dir;      /* direction k of each term */
    const int64_t* term_node;     /* pitched node y of each term */
    const int32_t* term_export;   /* AA: export index holding f*_k(y) */
    const void* term_coeff;       /* real[n_terms] */
    const void* local_force;      /* real[d][n_local] immersed-boundary node force */
    int32_t n_local;
    int32_t n_export;
    const void* export_in;        /* AA: real[n_export] written by the previous launch */
    void* export_out;             /* AA: real[n_export] read by the next launch */
} lbm_special_t;

/* Bulk tiling of a step launch: tile_x * tile_y threads per block, one node each. */
typedef struct lbm_launch {
    int32_t tile_x;   /* multiple of 32 */
    int32_t tile_y;
} lbm_launch_t;

/* ---- the time step ---------------------------------------------------- */

/* Two-lattice fused pull stream + bounce-back + link rules + TRT/Guo collide.
 * Replaces the reference kernel stream_collide_naive
 * (src/lbm/backends/kernels/stream_collide_naive.cu:15-49) together with its
 * rule pre-pass rules_evaluate/rules_write (kernels/link_rules.cu:15-43,
 * launched from src/lbm/backends/cuda_solver.py:157-176). f_src is read only;
 * f_dst receives every fluid node (solid nodes are left untouched). */
int lbm_step_pull(const lbm_grid_t* grid, const lbm_physics_t* phys, const lbm_special_t* sp,
                  const lbm_launch_t* launch, const uint8_t* kind, const void* f_src, void* f_dst,
                  lbm_stream_t stream);

/* In-place AA step (Bailey et al. 2009) on one lattice; parity LBM_AA_ODD or
 * LBM_AA_EVEN. Replaces aa_odd / aa_even (kernels/stream_collide_aa.cu:33-98)
 * and their rule pre-passes. Rules read sp->export_in and exporter nodes
 * write sp->export_out; the caller swaps the two after every launch. */
int lbm_step_aa(const lbm_grid_t* grid, const lbm_physics_t* phys, const lbm_special_t* sp,
                const lbm_launch_t* launch, const uint8_t* kind, void* f, int32_t parity,
                lbm_stream_t stream);

/* Fill the AA export buffer from a stored state in the given layout (after
 * initialisation or an external write of the populations). */
int lbm_export_prime(const lbm_grid_t* grid, const lbm_special_t* sp, const void* f, int32_t layout,
                     void* export_out, lbm_stream_t stream);

/* ---- node kinds -------------------------------------------------------- */

/* kind[node] = SOLID | SPECIAL | NEAR from a solid mask (uint8, 0/1, pitched
 * like the lattice) and a list of special nodes. Periodic neighbours. */
int lbm_classify(const lbm_grid_t* grid, const uint8_t* solid, const int64_t* special_nodes,
                 int32_t n_special, uint8_t* kind, lbm_stream_t stream);

/* ---- state conversion ------------------------------------------------- */

/* Equilibrium state from float64 density and velocity fields (pitched):
 * u' = u + F/(2 rho) with F = phys->force + phys->force_field, combined in
 * float64 and cast once to the compute type, then the shifted equilibrium --
 * replaces Solver._initial_populations (src/lbm/solver.py:101-117). layout
 * selects the stored slot order (LBM_LAYOUT_AA_ODD stores f*_i in slot
 * opp(i), cuda_solver.py:260-262). Every node is written, solid ones too. */
int lbm_init_equilibrium(const lbm_grid_t* grid, const lbm_physics_t* phys, const double* rho,
                         const double* u, int32_t layout, void* f, lbm_stream_t stream);

/* Natural-order populations in the compute type: out[i][node] = f*_i(node);
 * replaces CudaSolver._device_populations (cuda_solver.py:302-305). */
int lbm_unpack(const lbm_grid_t* grid, const void* f, int32_t layout, void* out, lbm_stream_t stream);

/* Inverse of lbm_unpack (population-exact restore from natural order). */
int lbm_pack(const lbm_grid_t* grid, const void* in, int32_t layout, void* f, lbm_stream_t stream);

/* ---- readouts --------------------------------------------------------- */

/* rho = 1 + sum f~*, rho u = sum c f* - F/2 with F = uniform + per-node field +
 * immersed-boundary force; solid nodes report rho = 1, u = 0. Replaces
 * Solver.macroscopic (src/lbm/solver.py:209-221, diagnostics.py:72-80).
 * Outputs real[nodes] and real[d][nodes], pitched. local_force may be NULL. */
int lbm_macroscopic(const lbm_grid_t* grid, const lbm_physics_t* phys, const uint8_t* kind,
                    const void* f, int32_t layout, const int64_t* local_nodes, const void* local_force,
                    int32_t n_local, void* rho, void* u, lbm_stream_t stream);

/* Divergence watchdog -- replaces Solver._check_health (src/lbm/solver.py:162-172).
 * out[0] = smallest pitched index of a fluid node with non-finite populations
 * or rho <= 0 (INT64_MAX if none); out[1] = 1 if any node is non-finite.
 * out must be zeroed with lbm_health_reset first (same stream). */
int lbm_health_reset(int64_t* out, lbm_stream_t stream);
int lbm_health(const lbm_grid_t* grid, const uint8_t* kind, const void* f, int64_t* out,
               lbm_stream_t stream);

/* Affine gather: values[r] = const[r] + sum_t coeff[r*n_terms+t] * f[slot[r*n_terms+t]]
 * in float64 over raw storage slots -- replaces Solver.evaluate_affine /
 * link_rules.evaluate_affine (src/lbm/solver.py:178-188, link_rules.py:269-272). */
int lbm_affine_gather(int32_t storage, const void* f, const int64_t* slots, const double* coeff,
                      const double* constant, int64_t n_rows, int32_t n_terms, double* values,
                      lbm_stream_t stream);

/* Momentum-exchange force: out[a] += sum_r weight[r*d+a] * value_r, value_r as
 * in lbm_affine_gather, reduced in float64 with warp shuffles -- replaces the
 * host matvec of ForceProbe.evaluate (src/lbm/forces.py:98-103). partial must
 * hold ceil(n_rows/256)*d doubles and counter one zeroed uint32; out is
 * overwritten (deterministic order). */
int lbm_affine_reduce(int32_t storage, const void* f, const int64_t* slots, const double* coeff,
                      const double* constant, const double* weight, int64_t n_rows, int32_t n_terms,
                      int32_t d, double* partial, uint32_t* counter, double* out, lbm_stream_t stream);

/* ---- immersed boundary (direct forcing, multi-direct) ------------------- */
/* Replaces ImmersedForcing.force_field (src/lbm/ibm.py:189-214). */

typedef struct lbm_ibm {
    int32_t n_nodes;           /* unique stencil nodes */
    int32_t n_markers;
    int32_t stencil_size;      /* 9 (2D) or 27 (3D) */
    const int64_t* node;       /* pitched index of each stencil node */
    const int32_t* stencil;    /* [n_markers][stencil_size] positions in node[] */
    const void* weight;        /* real[n_markers][stencil_size] Roma weights */
    const void* area;          /* real[n_markers] */
    const int32_t* inv_start;  /* [n_nodes + 1] CSR over (marker, weight) pairs per node */
    const int32_t* inv_marker;
    const void* inv_weight;    /* real */
    void* rho;                 /* real[n_nodes] scratch */
    void* u_star;              /* real[d][n_nodes] scratch */
    void* marker_force;        /* real[iterations][d][n_markers]: F_l of every pass */
} lbm_ibm_t;

/* Moments of the streamed populations at the stencil nodes (state in layout). */
int lbm_ibm_moments(const lbm_grid_t* grid, const lbm_physics_t* phys, const lbm_ibm_t* ibm,
                    const void* f, int32_t layout, lbm_stream_t stream);

/* One multi-direct pass: force_out = force_in + spread of the marker forces
 * computed from u* + force_in / (2 rho). force_in may be NULL (first pass). */
int lbm_ibm_iteration(const lbm_grid_t* grid, const lbm_ibm_t* ibm, int32_t iteration,
                      const void* force_in, void* force_out, lbm_stream_t stream);

/* Body force -sum_iterations sum_l F_l in float64 (out[d]). */
int lbm_ibm_body_force(const lbm_grid_t* grid, const lbm_ibm_t* ibm, int32_t iterations, double* out,
                       lbm_stream_t stream);

/* ---- diagnostics ------------------------------------------------------- */

/* Registers, local (spill) bytes, static shared bytes and max threads per
 * block of one step kernel; replaces CudaSolver.kernel_resources
 * (cuda_solver.py:311-326). which = LBM_PULL / LBM_AA_EVEN / LBM_AA_ODD. */
int lbm_kernel_resources(int32_t lattice, int32_t storage, int32_t which, int32_t* out4);

/* Name of the last CUDA error seen by the library in this thread (static string). */
const char* lbm_last_cuda_error(void);

/* Library ABI version (bumped on any incompatible change). */
int32_t lbm_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
