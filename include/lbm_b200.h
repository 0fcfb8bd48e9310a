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
    LBM_ERR_LAUNCH = -3,       /* kernel launch failed; see lbm_last_cuda_error */
    LBM_ERR_TOO_LARGE = -4     /* size beyond a fixed in-library scratch limit */
};

/* ---- enums ------------------------------------------------------------ */
enum { LBM_D2Q9 = 0, LBM_D3Q19 = 1 };
enum { LBM_F32 = 0, LBM_F64 = 1, LBM_F16 = 2, LBM_BF16 = 3 };
enum { LBM_PULL = 0, LBM_AA_EVEN = 1, LBM_AA_ODD = 2 };
/* Collision model (lbm_physics_t.collision). TRT covers BGK (omega_minus == omega_plus).
 * REGULARIZED: projective regularisation of the non-equilibrium part onto the
 * second-order Hermite moments (Latt & Chopard 2006) before a single-rate
 * relaxation with omega_plus, Guo forcing -- not in the reference (its roadmap
 * item 3, README "High Reynolds numbers"); the one-node kernels run it
 * whatever the storage, the adjoint and batched steps take TRT only.
 * CUMULANT (D2Q9 only): the cumulant method (Geier et al. 2015) on the
 * tensor-product lattice -- central moments about u = (j + F/2)/rho by the
 * chimera transformation, shear moments relaxed with omega_plus, bulk,
 * third-order and the fourth-order cumulant relaxed with rate 1, first-order
 * moments mirrored (the force); also one-node kernels only, not in the adjoint
 * or batched steps; LBM_ERR_UNSUPPORTED on D3Q19. */
enum { LBM_COLLIDE_TRT = 0, LBM_COLLIDE_REGULARIZED = 1, LBM_COLLIDE_CUMULANT = 2 };
/* Where a stored state keeps f*_k(y) (reference src/lbm/link_rules.py:16-25). */
enum { LBM_LAYOUT_PULL = 0, LBM_LAYOUT_AA_ODD = 1, LBM_LAYOUT_AA_EVEN = 2 };
/* Node kind bits (one byte per node): SOLID; SPECIAL (updated by the boundary
 * warps); NEAR (fluid with a solid neighbour); EDGE (fluid on a face of the
 * box, neighbours wrap periodically). Kind 0 = interior fluid node. */
enum { LBM_KIND_SOLID = 1, LBM_KIND_SPECIAL = 2, LBM_KIND_NEAR = 4, LBM_KIND_EDGE = 8 };

/* ---- descriptors ------------------------------------------------------ */
typedef struct lbm_grid {
    int32_t lattice;   /* LBM_D2Q9 or LBM_D3Q19 */
    int32_t storage;   /* LBM_F32, LBM_F64, LBM_F16, LBM_BF16 */
    int32_t nx, ny, nz;
    int32_t pitch;     /* row pitch in nodes, >= nx */
    int64_t qstride;   /* elements between direction planes, >= pitch * ny * nz */
} lbm_grid_t;

/* Collision constants and wall data. "real" arrays use the compute type:
 * double for LBM_F64 storage, float otherwise. */
typedef struct lbm_physics {
    double omega_plus;     /* 1/tau */
    double omega_minus;    /* TRT antisymmetric rate (== omega_plus for BGK) */
    double force[3];       /* uniform body-force density */
    const void* wall_u;    /* real[d][qstride] wall velocity at solid nodes, or NULL (all walls at rest) */
    const void* force_field; /* real[d][qstride] per-node body force added to force[], or NULL */
    const uint32_t* solid_nbr; /* per node: bit i set where x - c_i is solid (lbm_classify); read only
                                  at fluid nodes that are not interior */
    int32_t collision;     /* LBM_COLLIDE_* */
    uint32_t* round_seed;  /* float16/bfloat16 storage (required there, ignored otherwise): three
                              uint32 slots in device memory. Slots 0 and 1 hold the step counter of
                              the stochastic rounding of stored populations: a step reads slot p and
                              its bulk (or fused) launch writes slot 1 - p with the count + 1, where
                              p = (f_src > f_dst) for lbm_step_pull and p = parity for lbm_step_aa.
                              Set both to the same value (0) whenever the populations are set.
                              Slot 2 is a status word, zeroed by the caller: the TMA-staged pull
                              kernel sets bit 0 when a block gave up waiting for its staged loads
                              (bounded wait), in which case the step's output is incomplete. */
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
    /* Optional dense form of the same rules (ut_start NULL: term by term).
     * The rules of special node s read the distinct populations
     * u in [ut_start[s], ut_start[s+1]) -- at most LBM_DENSE_TERMS -- and rule r
     * of that node is  const[r] + sum_u rule_dense[rule_row[r] + u - ut_start[s]] * value(u),
     * so each distinct population is loaded once for all the node's rules
     * (a Zou-He node's five rules share its fourteen known populations). */
    const int32_t* ut_start;      /* n_special + 1 */
    const int64_t* ut_slot;       /* pull: slot (dir * qstride + pitched node) of each distinct term */
    const int32_t* ut_export;     /* AA: export index of each distinct term */
    const int32_t* rule_row;      /* n_rules: start of rule r's row, a multiple of 4; the rows of one
                                     node's rules are consecutive, each (n + 3) & ~3 long (n: the node's
                                     distinct populations), and the kernels read the first one only */
    const void* rule_dense;       /* real, 16-byte aligned; rows zero-padded to multiples of 4 */
} lbm_special_t;

/* Distinct populations a special node's rules may read in the dense form. */
#define LBM_DENSE_TERMS 32

/* How a step is launched. The bulk grid covers every fluid node that is not
 * SPECIAL with blocks of tile_x * tile_y threads, one node each, over
 * (ceil(nx/tile_x), ceil(ny/tile_y), nz): interior nodes (kind 0) stream with
 * fixed offsets, nodes next to a wall or on a periodic face take the general
 * path driven by phys->solid_nbr. SPECIAL nodes (link rules, an
 * immersed-boundary force, AA exports) must be in the special list and are
 * updated by the boundary warps:
 *   LBM_LAUNCH_FUSED    one launch, boundary warps in extra z-planes of blocks;
 *   LBM_LAUNCH_BULK     the bulk grid only;
 *   LBM_LAUNCH_BOUNDARY the boundary warps only (1D grid over the list).
 * BULK and BOUNDARY touch disjoint nodes and may run concurrently; together
 * they are one time step. Split launches let the bulk kernel keep its small
 * register budget. For float16/bfloat16 storage, LBM_LAUNCH_BULK of
 * lbm_step_pull takes the TMA-staged kernel (persistent blocks over 2-row
 * tiles, tile_x/tile_y unused) when nx is a power of two in [32, 256], pitch
 * is a multiple of 16, f_src and kind are 16-byte aligned, force_field is
 * NULL and round_seed is given; otherwise a kernel with two nodes per thread
 * (pitch and qstride even, no force_field), else one node per thread. All
 * three give the same bits. lbm_step_aa chooses the same way, its TMA-staged
 * halves taking nx in [64, 256]. */
enum { LBM_LAUNCH_FUSED = 0, LBM_LAUNCH_BULK = 1, LBM_LAUNCH_BOUNDARY = 2 };

/* Health and mass check fused into a step (the step that ends a chunk of the
 * run loop) -- replaces the separate scan of Solver._check_health
 * (src/lbm/solver.py:162-172) over the state that step stores. Every fluid
 * node the launch updates checks its stored post-collision populations:
 * drho = sum_i f~*_i (direction order, the values as stored), bad if
 * non-finite or drho <= -1; and the launch sums f~* over its nodes in
 * float64, one partial sum per block, in a fixed order. */
typedef struct lbm_health {
    int64_t* words;      /* [0] smallest pitched index of a bad node (INT64_MAX: none), [1] 1 if a bad
                            node is non-finite; set both with lbm_health_reset before the step */
    double* partial;     /* n_partial doubles, written by the step (one per block) */
    int64_t n_partial;   /* exactly lbm_health_partials(grid, sp, launch) for the step's launch mode */
    void* rho;           /* NULL, or the macroscopic readout fused into the same step (reference
                            macroscopic_from_post_collision, src/lbm/diagnostics.py:72-80): rho (qstride)
                            and u (d, qstride) in the compute type, pitched, of every fluid node the
                            step updates, from the values it stores -- the bits lbm_macroscopic gives
                            for that state; solid nodes are left as they are (fill rho = 1, u = 0) */
    void* u;
} lbm_health_t;

typedef struct lbm_launch {
    int32_t tile_x;   /* multiple of 32 */
    int32_t tile_y;   /* tile_x * tile_y <= 256 */
    int32_t mode;     /* LBM_LAUNCH_* */
    uint32_t tma_wait_limit; /* TMA-staged kernels: polls of the wait for a tile's staged loads before
                                the block gives up (status word bit 0, see round_seed); 0 = the default,
                                2^22 polls; LBM_TMA_WAIT_NONE = no poll at all, so every block gives up
                                at its first tile (to exercise the time-out path). The block's final
                                wait for loads still in flight always takes the default, so that none
                                is left in flight when it exits. */
    const lbm_health_t* health; /* NULL: a plain step. Else a checked step (lbm_step_pull, or lbm_step_aa
                                   with parity LBM_AA_EVEN; LBM_ERR_INVALID for the odd half): the bulk
                                   launch takes the one-node kernel whatever the storage (all bulk
                                   kernels give the same bits); split launches (BULK + BOUNDARY) take
                                   the same lbm_health_t and fill disjoint partial slots. */
} lbm_launch_t;
#define LBM_TMA_WAIT_NONE 0xFFFFFFFFu

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

/* kind[node] = SOLID | SPECIAL | NEAR | EDGE from a solid mask (uint8, 0/1, pitched
 * like the lattice) and a list of special nodes; solid_nbr[node] = bit i set
 * where node - c_i is solid (periodic neighbours), or NULL to skip it. */
int lbm_classify(const lbm_grid_t* grid, const uint8_t* solid, const int64_t* special_nodes,
                 int32_t n_special, uint8_t* kind, uint32_t* solid_nbr, lbm_stream_t stream);

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

/* Partial slots a checked step with this launch writes (see lbm_health_t):
 * FUSED: one per block of the fused grid; BULK or BOUNDARY: the bulk grid's
 * blocks then the boundary launch's. Negative: invalid arguments. */
int64_t lbm_health_partials(const lbm_grid_t* grid, const lbm_special_t* sp, const lbm_launch_t* launch);

/* After a checked step (both launches, when split): delta_mass[0] = the sum of
 * h->partial[0 .. n_partial) in a fixed order, float64 -- the sum of f~* over
 * the fluid nodes, i.e. the mass minus the number of fluid nodes. */
int lbm_health_finish(const lbm_health_t* h, double* delta_mass, lbm_stream_t stream);

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

/* No-allocation variant of lbm_affine_reduce (no counterpart in the
 * reference, which reduces probe forces on the host). Same arguments, result
 * and summation order, minus partial and counter: the scratch is a fixed
 * array inside this library (96.25 KiB per device), so the call allocates
 * nothing and needs no buffers beyond its inputs and out[d].
 * For callers that cannot allocate device memory at the point of the call:
 * a C or Fortran host that owns only the lattice buffers and has no device
 * allocator, or a force readout between the launches of a running step loop,
 * where a cudaMalloc would synchronize the whole device.
 * Limit: n_rows <= LBM_AFFINE_REDUCE_STATIC_MAX_ROWS; a larger n_rows returns
 * LBM_ERR_TOO_LARGE and launches nothing (use lbm_affine_reduce instead).
 * Set-up: the first call on each device, made with that device current,
 * looks up the array's address and caches it (this may load the library's
 * device code); make that first call before any stream capture. The cache
 * belongs to the device's current context: after cudaDeviceReset the first
 * call in the new context looks the address up again (same rule on capture).
 * Calls share one array per device: calls that may overlap in time on the
 * same device (different streams, or host threads without ordering) race
 * and give wrong sums; issue them on one stream. Each call clears the block
 * counter on its stream before the reduction. */
#define LBM_AFFINE_REDUCE_STATIC_MAX_ROWS 1048576
int lbm_affine_reduce_static(int32_t storage, const void* f, const int64_t* slots, const double* coeff,
                             const double* constant, const double* weight, int64_t n_rows, int32_t n_terms,
                             int32_t d, double* out, lbm_stream_t stream);

/* ---- device-side rule compiler ------------------------------------------ */
/* The geometry and link-rule tables of the host builders, built on the device
 * from the solid mask (uint8 0/1, pitched like the lattice) and the body: for a
 * 256^3 grid with a sphere the host's voxelisation and wall-link search take
 * tens of seconds. Node indices in and out are natural (unpitched) flat
 * indices ((z ny + y) nx + x), as the host builders use. Every floating-point
 * operation follows the host's order with explicit IEEE rounding, so the
 * results equal the host builders' bit for bit. A ball is its centre (cz
 * ignored in 2D) and squared radius. */

/* solid[node] = 1 at every node inside the ball -- replaces voxelize(body, shape)
 * for a ball (src/lbm/geometry.py:140-144, 74-76). */
int lbm_ball_voxelize(const lbm_grid_t* grid, double cx, double cy, double cz, double radius_sq, uint8_t* solid,
                      lbm_stream_t stream);

/* Every link (x, j) from a fluid node x into the ball (x - c_j inside, periodic
 * wrap), ordered by direction j then node, with the wall fraction q along the
 * link (first root of |x - t c_j - centre| = R, clipped to (0, 1]) -- replaces
 * wall_links(lattice, body, solid) (src/lbm/geometry.py:174-206, 78-87).
 * Two passes over a scratch of lbm_ball_links_scratch(grid) int64 (with
 * m = Q * ceil(qstride / 256) per-(direction, block) counts in front):
 * lbm_ball_links_count leaves the link count in scratch[m] and the number of
 * nodes inside the ball that are not solid (must be 0) in scratch[m + 1];
 * lbm_ball_links_write (same arguments and scratch) fills node[count],
 * direction[count], q[count]. */
int64_t lbm_ball_links_scratch(const lbm_grid_t* grid);
int lbm_ball_links_count(const lbm_grid_t* grid, const uint8_t* solid, double cx, double cy, double cz,
                         double radius_sq, int64_t* scratch, lbm_stream_t stream);
int lbm_ball_links_write(const lbm_grid_t* grid, const uint8_t* solid, double cx, double cy, double cz,
                         double radius_sq, const int64_t* scratch, int64_t* node, int32_t* direction, double* q,
                         lbm_stream_t stream);

/* The Bouzidi rule of each link -- replaces bouzidi_rules (src/lbm/link_rules.py:154-188):
 * with i = opp(j), link r gets two terms (term_dir/term_node/coeff[2r], [2r + 1]):
 * q < 1/2: 2q f*_i(x) + (1 - 2q) f*_i(x + c_j); q >= 1/2: f*_i(x)/(2q) + (1 - 1/(2q)) f*_j(x);
 * keep[r] = 0 where q < 1/2 and x + c_j is solid (the link keeps plain bounce-back). */
int lbm_bouzidi_links(const lbm_grid_t* grid, const uint8_t* solid, int64_t n, const int64_t* node,
                      const int32_t* direction, const double* q, uint8_t* keep, int64_t* term_dir,
                      int64_t* term_node, double* coeff, lbm_stream_t stream);

/* Slots of affine terms f*_k(y) in a stored layout, pitched for this library's
 * buffers (slot = direction plane * qstride + pitched node) -- replaces the slot
 * resolution of compile_affine (src/lbm/link_rules.py:203-240): LBM_LAYOUT_PULL
 * (k, y); LBM_LAYOUT_AA_ODD (opp k, y); LBM_LAYOUT_AA_EVEN (k, y + c_k), or
 * (opp k, y) where y + c_k is solid, with extra[t] = coeff[t] 6 w_k (c_k . u_w(y + c_k))
 * (wall_u: float64 (d, qstride) pitched, or NULL: extra is 0) to add to the row's
 * constant. solid is needed for LBM_LAYOUT_AA_EVEN only; extra may be NULL. */
int lbm_compile_terms(const lbm_grid_t* grid, int32_t layout, const uint8_t* solid, const double* wall_u, int64_t n,
                      const int64_t* direction, const int64_t* node, const double* coeff, int64_t* slot,
                      double* extra, lbm_stream_t stream);

/* Zou-He velocity inlet / density outlet rules of one open column x = column of a
 * channel whose x = 0 and x = nx - 1 layers are closed -- replaces _zou_he and
 * open_channel (src/lbm/open_boundaries.py:96-186). solid: the closed mask
 * (natural order, pitch = nx); layer: (nz * ny) the fluid nodes of the open
 * layer at x = layer_x before it was closed; sign +1: inlet, velocity (d, nz * ny)
 * prescribed at the column; sign -1: outlet at density rho_out (velocity NULL;
 * LBM_ERR_INVALID for an inlet without a velocity or an outlet with one).
 * Node (x, y, z) of the column gets one rule per unknown population j
 * (sign c_jx = +1, ascending j) when it is fluid and some unknown streams in from
 * the layer: f_j = b + sum a_m f*_{k_m}(y_m), its non-zero terms over the node's
 * streamed populations packed to the front in ascending k, b the shifted-storage
 * constant. Two passes over a scratch of lbm_zou_he_scratch(grid) int64 (n = ny * nz):
 * lbm_zou_he_count leaves the number of nodes with rules in scratch[n] and the
 * largest number of terms of a rule in scratch[n + 1]; lbm_zou_he_write (same
 * arguments and scratch) fills node[rows], direction[rows], term_dir/term_node/
 * coeff[rows][width] (zero beyond each rule's terms) and constant[rows], rows =
 * nodes * unknowns, node by node. */
int64_t lbm_zou_he_scratch(const lbm_grid_t* grid);
int lbm_zou_he_count(const lbm_grid_t* grid, const uint8_t* solid, int32_t column, int32_t sign, int32_t layer_x,
                     const uint8_t* layer, const double* velocity, double rho_out, int64_t* scratch,
                     lbm_stream_t stream);
int lbm_zou_he_write(const lbm_grid_t* grid, const uint8_t* solid, int32_t column, int32_t sign, int32_t layer_x,
                     const uint8_t* layer, const double* velocity, double rho_out, const int64_t* scratch,
                     int32_t width, int64_t* node, int64_t* direction, int64_t* term_dir, int64_t* term_node,
                     double* coeff, double* constant, lbm_stream_t stream);

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
    const int32_t* inv_start;  /* [n_nodes + 1] CSR over (marker, weight) pairs per node; every
                                  (marker, stencil position) appears once: inv_start[n_nodes] ==
                                  n_markers * stencil_size */
    const int32_t* inv_marker;
    const void* inv_weight;    /* real */
    void* rho;                 /* real[n_nodes] scratch */
    void* u_star;              /* real[d][n_nodes] scratch */
    void* marker_force;        /* real[iterations][d][n_markers]: F_l of every pass */
    double* marker_scratch;    /* (1 + 2 d) doubles per marker for lbm_ibm_adjoint_iteration (each marker's
                                  terms formed once, then read by its nodes), or NULL (each node forms the
                                  terms of its markers itself); same results either way */
} lbm_ibm_t;

/* Moments of the streamed populations at the stencil nodes (state in layout). */
int lbm_ibm_moments(const lbm_grid_t* grid, const lbm_physics_t* phys, const lbm_ibm_t* ibm,
                    const void* f, int32_t layout, lbm_stream_t stream);

/* One multi-direct pass: force_out = force_in + spread of the marker forces
 * computed from u* + force_in / (2 rho). force_in may be NULL (first pass).
 * Two launches: the marker forces (into marker_force[iteration]), then the
 * node-centric spread. */
int lbm_ibm_iteration(const lbm_grid_t* grid, const lbm_ibm_t* ibm, int32_t iteration,
                      const void* force_in, void* force_out, lbm_stream_t stream);

/* The immersed-boundary node force of one step in one call: moments of the
 * state f (in layout) and `iterations` multi-direct passes -- replaces the
 * array code of ImmersedForcing.force_field (src/lbm/ibm.py:189-214, run
 * before every step by src/lbm/solver.py). force: real[iterations][d][n_nodes],
 * pass j written to force[j] (the last pass is the node force the step adds);
 * marker forces of every pass in ibm->marker_force as lbm_ibm_iteration.
 * Bodies of up to 4096 stencil nodes and markers run as one one-block launch;
 * larger ones as lbm_ibm_moments + one lbm_ibm_iteration launch per pass. */
int lbm_ibm_force(const lbm_grid_t* grid, const lbm_physics_t* phys, const lbm_ibm_t* ibm, const void* f,
                  int32_t layout, int32_t iterations, void* force, lbm_stream_t stream);

/* The immersed-boundary part of one pull step in one launch: lbm_ibm_force of
 * f_src (layout LBM_LAYOUT_PULL, into force as there), then, in the same
 * block, the step of the special nodes in sp -- the body's stencil nodes --
 * from f_src into f_dst with the final pass's node force (sp->local_force and
 * sp->n_local are set to it; force_slot indexes it), exactly as a
 * LBM_LAUNCH_BOUNDARY launch of lbm_step_pull would update them. With the
 * step's other special nodes in a BOUNDARY launch and the bulk in a BULK
 * launch, all three concurrent, no launch of the step waits for the force
 * (replaces lbm_ibm_force followed by a BOUNDARY launch over every special
 * node; reference src/lbm/solver.py runs the force before each step,
 * src/lbm/ibm.py:189-214). Bodies of up to 4096 stencil nodes and markers;
 * larger ones return LBM_ERR_UNSUPPORTED. */
int lbm_step_pull_ibm(const lbm_grid_t* grid, const lbm_physics_t* phys, const lbm_special_t* sp,
                      const lbm_ibm_t* ibm, int32_t iterations, const uint8_t* kind, const void* f_src,
                      void* f_dst, void* force, lbm_stream_t stream);

/* Body force -sum_iterations sum_l F_l in float64 (out[d]). */
int lbm_ibm_body_force(const lbm_grid_t* grid, const lbm_ibm_t* ibm, int32_t iterations, double* out,
                       lbm_stream_t stream);

/* Reverse of one multi-direct pass (no counterpart in the reference, which has
 * no adjoint). With the forward quantities of the step recomputed in ibm
 * (rho, u_star, and force_prev = the node force entering the pass, NULL for
 * the first), adj_in = dL/d(node force after the pass), and the body-force
 * loss term dL/dF_l[axis] = -body_scale (axis < 0: none), node-centric:
 *   Fbar_l  = sum_s w_ls adj_in(m(l,s)) - body_scale e_axis
 *   adj_out(n)     = adj_in(n) - (1/rho_n) sum_l dA_l rho_l w_ln Fbar_l   (if adj_out != NULL)
 *   moment_adj[1+a](n) += sum_l -2 dA_l rho_l w_ln Fbar_l[a]             (dL/du*)
 *   moment_adj[0](n)   += sum_l w_ln (-2 dA_l U_l . Fbar_l)
 *                         + dA_l rho_l w_ln (Fbar_l . force_prev(n)) / rho_n^2   (dL/drho)
 * moment_adj: double[1 + d][n_nodes], accumulated over the passes. */
int lbm_ibm_adjoint_iteration(const lbm_grid_t* grid, const lbm_ibm_t* ibm, const void* force_prev,
                              const void* adj_in, int32_t axis, double body_scale, void* adj_out,
                              double* moment_adj, lbm_stream_t stream);

/* Closing part of the immersed-boundary adjoint (no counterpart in the
 * reference): dL/d(streamed populations) at the stencil nodes from moment_adj,
 *   mu[k](n) += rho_bar_n + c_k . u*_bar_n / rho_n,
 *   rho_bar_n = moment_adj[0](n) - u*_bar_n . u*_n / rho_n,
 * added into mu (real[Q][qstride], the adjoint of the streamed state written
 * by lbm_adjoint_step); moment_adj is then zeroed for the next step. */
int lbm_ibm_adjoint_moments(const lbm_grid_t* grid, const lbm_ibm_t* ibm, double* moment_adj, void* mu,
                            lbm_stream_t stream);

/* ---- adjoint (reverse mode) of the two-lattice step ---------------------- */

/* Extra tables of the adjoint step, per node of the adjoint special list (the
 * forward list plus every node that a rule term or the loss reads).
 *   gather[g] for g in [gather_start[s], gather_start[s+1]): direction k of
 *   the node and a contribution coeff * mu[slot] (slot >= 0) or coeff * loss_scale
 *   (slot < 0, the loss gradient of a force probe) to lambda_k(node). */
typedef struct lbm_adjoint {
    const int32_t* gather_start;   /* n_special + 1 */
    const int32_t* gather_dir;
    const int64_t* gather_slot;    /* slot of mu (k * qstride + pitched node) or -1 */
    const void* gather_coeff;      /* real */
    const void* rule_dconst;       /* real[n_rules]: d const / dU of each rule, or NULL */
    const void* term_dcoeff;       /* real[n_terms]: d coeff / dU aligned with the rule terms */
    double* rule_du;               /* double[n_rules] accumulator: sum over steps of mu_j * d rule value / dU */
    void* force_grad;              /* real[d][qstride] accumulator of dL/dG, or NULL */
    void* local_force_grad;        /* real[d][n_local]: dL/dF at each special node with a force slot
                                      (sp->force_slot >= 0, the immersed-boundary stencil nodes, whose
                                      collision adds sp->local_force), written by every step, or NULL */
    const void* rule_ddense;       /* real: d coeff / dU in the layout of sp->rule_dense (with sp->ut_start
                                      set and rule_du wanted), or NULL: rules are evaluated term by term */
} lbm_adjoint_t;

/* One backward step of the two-lattice pull scheme, fused:
 *   lambda_{t+1}(x) = reverse-pull of mu_next (bounce-back and link rules
 *       transposed) + loss_scale * dD/df at probe slots;
 *   s_t(x) = streamed populations of f_t (recomputed, as the forward step);
 *   mu_t(x) = J_C(s_t(x), F(x))^T lambda_{t+1}(x)       -> mu_out
 *   force_grad(x) += J_F^T lambda_{t+1}(x); rule_du += mu_j * d value / dU.
 * mu_next may be NULL (lambda_T = loss_scale * dD/df). Traffic: read f_t and
 * mu_next, write mu_out (3 Q values per node). Same launch modes as the step. */
int lbm_adjoint_step(const lbm_grid_t* grid, const lbm_physics_t* phys, const lbm_special_t* sp,
                     const lbm_adjoint_t* adj, const lbm_launch_t* launch, const uint8_t* kind,
                     const void* f_t, const void* mu_next, void* mu_out, double loss_scale,
                     lbm_stream_t stream);

/* Closing term: lambda_0 = reverse-pull of mu_0, and force_grad += the
 * derivative of the initial equilibrium (velocity shifted by F/(2 rho), F
 * including the per-node force) w.r.t. the per-node force. rho0/u0: the
 * float64 fields the state was initialised from (pitched). */
int lbm_adjoint_initial(const lbm_grid_t* grid, const lbm_physics_t* phys, const lbm_special_t* sp,
                        const lbm_adjoint_t* adj, const uint8_t* kind, const void* mu0, const double* rho0,
                        const double* u0, double loss_scale, lbm_stream_t stream);

/* ---- batched domains (many independent lattices, one launch per step) ---- */

/* One domain of a batch: a lattice of its own in pooled buffers. */
typedef struct lbm_domain {
    int32_t nx, ny, nz, pitch;
    int64_t offset;        /* element offset of the domain's direction-0 plane in the population pools */
    int64_t qstride;       /* pitch * ny * nz */
    int64_t kind_offset;   /* byte offset of the domain's kind array in the kind pool */
    int64_t wall_offset;   /* element offset of its wall velocity (d planes of qstride) or -1 */
    double omega_plus, omega_minus;
    double force[3];
} lbm_domain_t;

/* Work list of a batch step: n_tiles tiles, each int32 x4 = (domain, tile
 * index along x, tile index along y, z). A persistent grid of `blocks` blocks
 * walks the tiles round-robin; no block waits for another. Every fluid node
 * of a tile is updated (interior path, or the general path for nodes next to
 * a wall or on a periodic face). */
typedef struct lbm_batch {
    int32_t lattice, storage;
    int32_t n_domains;
    const lbm_domain_t* domains;   /* device array */
    int32_t n_tiles;
    const int32_t* tiles;          /* device, 4 int32 per tile */
    int32_t tile_x, tile_y;        /* tile_x multiple of 32, tile_x * tile_y <= 256 */
    int32_t blocks;                /* persistent grid size (> 0) */
    const uint8_t* kind;           /* kind pool (domain i at kind_offset) */
    const uint32_t* solid_nbr;     /* solid-neighbour pool, same offsets as kind */
    const void* wall_u;            /* wall pool (compute type) or NULL */
    uint32_t* round_seed;          /* slots 0 and 1 as lbm_physics_t.round_seed, one counter for the
                                      whole batch (slot 2 is not used here) */
} lbm_batch_t;

/* One two-lattice pull step of every domain of the batch -- the batched
 * counterpart of lbm_step_pull (no link rules or immersed bodies). */
int lbm_batch_step(const lbm_batch_t* batch, const void* f_src, void* f_dst, lbm_stream_t stream);

/* Blocks of the batch kernel that fit on one SM for the given tile (occupancy
 * API), for sizing the persistent grid. */
int lbm_batch_occupancy(int32_t lattice, int32_t storage, int32_t tile_x, int32_t tile_y, int32_t* blocks_per_sm);

/* ---- diagnostics ------------------------------------------------------- */

/* Registers, local (spill) bytes, static shared bytes and max threads per
 * block of one step kernel; replaces CudaSolver.kernel_resources
 * (cuda_solver.py:311-326). which = variant + 3 * launch mode
 * (variant LBM_PULL / LBM_AA_EVEN / LBM_AA_ODD, mode LBM_LAUNCH_*). */
int lbm_kernel_resources(int32_t lattice, int32_t storage, int32_t which, int32_t* out4);

/* Name of the last CUDA error seen by the library in this thread (static string). */
const char* lbm_last_cuda_error(void);

/* Library ABI version (bumped on any incompatible change). */
int32_t lbm_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
