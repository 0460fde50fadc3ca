/* glide_b200.h -- C ABI of the B200-native SSA momentum + mass-conservation
 * solver (drop-in for the hot path of JacobDowns/glide).
 *
 * Plain pointers and sizes only.  Device pointers are CUDA device addresses;
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 * Every function returns GLIDE_OK (0) or an error code; glide_last_error()
 * gives the message of the last failure on the calling thread.  A handle is
 * not thread-safe: use one handle per host thread.
 *
 * Reference interfaces each entry point replaces (paths inside the
 * JacobDowns/glide project):
 *   glide_create / glide_destroy   glide/multigrid.py:8-52 Multigrid.__init__ (+ grid.py:147-233)
 *   glide_field_ptr                Field.data of every level (glide/field.py:41-61, grid.py:235-350)
 *   glide_set_field                HierarchyFieldManager.set (glide/multigrid.py:271-274)
 *   glide_restrict_field           HierarchyFieldManager.restrict_down (glide/multigrid.py:276-280)
 *   glide_get_field                reading Field.data / Field.grad
 *   glide_set_phys / get_phys      Constant fields of Geometry/Rheology/Sliding/Calving (grid.py:8-145)
 *   glide_set_fas_config           FASCDOptions.set / FASAdjointOptions.set (glide/multigrid.py:767-777, :1045-1049)
 *   glide_set_vanka_config         VankaOptions / NewtonOptions .set / .set_level (glide/multigrid.py:780-852)
 *   glide_set_rhs                  ForwardOperators.set_rhs (glide/operators.py:275-276)
 *   glide_compute_phi              ForwardOperators.compute_phi (glide/operators.py:173-192)
 *   glide_residual                 ForwardOperators.compute_residual (glide/operators.py:71-127)
 *   glide_vanka_sweep              ForwardOperators.vanka_sweep (glide/operators.py:243-251)
 *   glide_forward                  FASCDSolver.solve (glide/multigrid.py:502-533) as called by
 *                                  IceDynamics.forward (glide/model.py:65-72)
 *   glide_adjoint_residual         AdjointOperators.compute_residual (glide/operators.py:379-425)
 *   glide_vjp                      AdjointOperators.compute_vjp (glide/operators.py:429-472)
 *   glide_adjoint_sweep            AdjointOperators.vanka_sweep (glide/operators.py:517-524)
 *   glide_gradients                AdjointOperators.compute_gradient_* (glide/operators.py:526-593)
 *   glide_backward                 IceDynamics.backward (glide/model.py:74-94) with
 *                                  FASAdjointSolver.solve (glide/multigrid.py:873-903)
 *   glide_vcycle                   FASCDSolver.vcycle / FASAdjointSolver.vcycle
 *                                  (glide/multigrid.py:536-645, :905-973)
 *   glide_transfer                 Multigrid.restrict_* / prolongate_* (glide/multigrid.py:119-259)
 */
#ifndef GLIDE_B200_H
#define GLIDE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define GLIDE_OK 0
#define GLIDE_ERR_ARG 1        /* bad argument (level, field, flag, null pointer) */
#define GLIDE_ERR_SHAPE 2      /* grid size not divisible by 2^(levels-1), or unsupported shape */
#define GLIDE_ERR_CUDA 3       /* a CUDA call failed */
#define GLIDE_ERR_NONFINITE 4  /* residual norm became NaN or Inf */
#define GLIDE_ERR_STATE 5      /* call not valid in the handle's current state */
/* glide_forward / glide_backward stopped at maximum_vcycles short of both
 * tolerances; returned only when GLIDE_TUNE_REPORT_NOT_CONVERGED is on (the
 * reference reports nothing), after every output and *stats is written. */
#define GLIDE_ERR_NOT_CONVERGED 6
#define GLIDE_ERR_TIMEOUT 7    /* a kernel's bounded wait (for its staged tile copies) gave up */

#define GLIDE_F64 0
#define GLIDE_F32 1
/* binary64 fields and residuals, binary32 smoother and coarse levels
 * (nonlinear defect correction); fields are accessed as binary64 */
#define GLIDE_MIXED 2

/* Field identifiers.  Face fields: U (ny, nx+1), V (ny+1, nx); all others are
 * cell fields (ny, nx).  ADJ_* are the adjoint operators' arrays, GRAD_* the
 * gradients written by glide_gradients / glide_backward, VJP_* the plain
 * transpose product written by glide_vjp, FOP_* the operator without forcing
 * written by glide_residual(GLIDE_OPERATOR_ONLY), VAR_* the direction and
 * JVP_* the Jacobian-vector product of glide_jvp. */
enum glide_field {
    GLIDE_U = 0, GLIDE_V, GLIDE_H, GLIDE_H_PREV, GLIDE_PHI, GLIDE_MASK,
    GLIDE_BED, GLIDE_B, GLIDE_BETA, GLIDE_SMB, GLIDE_GAMMA,
    GLIDE_F_U, GLIDE_F_V, GLIDE_F_H,
    GLIDE_R_U, GLIDE_R_V, GLIDE_R_H,
    GLIDE_LAMBDA_U, GLIDE_LAMBDA_V, GLIDE_LAMBDA_H,
    GLIDE_ADJ_F_U, GLIDE_ADJ_F_V, GLIDE_ADJ_F_H,
    GLIDE_ADJ_R_U, GLIDE_ADJ_R_V, GLIDE_ADJ_R_H,
    GLIDE_GRAD_BETA, GLIDE_GRAD_BED, GLIDE_GRAD_H_PREV, GLIDE_GRAD_SMB,
    GLIDE_VJP_U, GLIDE_VJP_V, GLIDE_VJP_H,
    GLIDE_FOP_U, GLIDE_FOP_V, GLIDE_FOP_H,
    GLIDE_VAR_U, GLIDE_VAR_V, GLIDE_VAR_H,
    GLIDE_JVP_U, GLIDE_JVP_V, GLIDE_JVP_H,
    GLIDE_N_PUBLIC_FIELDS
};

/* Flags of glide_residual / glide_vanka_sweep. */
#define GLIDE_USE_MASK 1
#define GLIDE_OPERATOR_ONLY 2
#define GLIDE_FREEZE_CALVING 4
#define GLIDE_FREEZE_PHI 8

/* Gradient selection of glide_gradients / glide_backward. */
#define GLIDE_GRAD_BETA_BIT 1
#define GLIDE_GRAD_BED_BIT 2
#define GLIDE_GRAD_H_PREV_BIT 4
#define GLIDE_GRAD_SMB_BIT 8

typedef struct glide_solver* glide_handle;

/* Physical constants of a level (defaults of glide/grid.py). */
typedef struct {
    double n, eps_reg, flotation_reg_driving, m, u_reg, water_drag,
        flotation_reg_sliding, calving_rate, flotation_reg_calving, thklim;
} glide_phys;

/* FASCD / FASAdjoint schedule (glide/multigrid.py:672-682, :993-1001). */
typedef struct {
    int freeze_coarse_calving, freeze_coarse_phi;
    int coarsest_steps, pre_steps, post_steps, finest_steps, maximum_vcycles;
    double relative_tolerance, absolute_tolerance;
} glide_fas_config;

/* Vanka smoother + local Newton (glide/operators.py:314-327).  `relaxation`
 * is stored but, as in the reference kernel, the local Newton uses 0.5. */
typedef struct {
    double omega;
    int newton_steps;
    double relaxation, ssa_damping, mc_damping, relax_phi;
} glide_vanka_config;

#define GLIDE_MAX_HISTORY 256
typedef struct {
    int vcycles;                     /* V-cycles run */
    double initial_norm, final_norm; /* sqrt(|r_u|^2+|r_v|^2+|r_H|^2) */
    double norms[3];                 /* final |r_u|, |r_v|, |r_H| */
    double history[GLIDE_MAX_HISTORY];
} glide_stats;

const char* glide_last_error(void);
int glide_version(void);

int glide_create(int ny, int nx, double dx, int n_levels, int dtype, glide_handle* out);
int glide_destroy(glide_handle h);
int glide_level_shape(glide_handle h, int level, int* ny, int* nx, double* dx);
int glide_field_ptr(glide_handle h, int field, int level, void** ptr, int* rows, int* cols,
                    int* pitch_elems);
int glide_set_field(glide_handle h, int field, int level, const void* src, int src_ld,
                    int src_on_host, int restrict_down, void* stream);
int glide_get_field(glide_handle h, int field, int level, void* dst, int dst_ld, int dst_on_host,
                    void* stream);
int glide_fill_field(glide_handle h, int field, int level, double value, int restrict_down,
                     void* stream);
int glide_restrict_field(glide_handle h, int field, int level, void* stream);
int glide_set_phys(glide_handle h, int level, const glide_phys* p);
int glide_get_phys(glide_handle h, int level, glide_phys* p);
/* `which`: 0 forward FASCD, 1 FASAdjoint, 2 tangent linear multigrid of the
 * Newton correction (no counterpart in the reference). */
int glide_set_fas_config(glide_handle h, int which, const glide_fas_config* c);
int glide_get_fas_config(glide_handle h, int which, glide_fas_config* c);
int glide_set_vanka_config(glide_handle h, int which, int level, const glide_vanka_config* c);
int glide_get_vanka_config(glide_handle h, int which, int level, glide_vanka_config* c);
/* on = 1 reproduces the reference's v-face prolongation (its u-face kernel
 * run on v arrays, glide/multigrid.py:212-235; square grids only). */
int glide_set_reference_quirks(glide_handle h, int on);
/* use_graphs = 1 replays each V-cycle as a captured CUDA graph. */
int glide_set_use_graphs(glide_handle h, int use_graphs);
/* Number of kernels this handle has launched so far (graph replays count
 * every kernel node; a GLIDE_MIXED handle's binary32 kernels included).
 * No counterpart in the reference: instrumentation. */
int glide_launch_count(glide_handle h, long long* count);
/* Algorithmic bytes of those kernels so far: for each launch, the values its
 * kernel must read and write once (N values per array of a level, face arrays
 * counted as N), plus the handle's device-to-device copies.  Divided by a
 * time it gives the achieved HBM bandwidth of a whole solve.  No counterpart
 * in the reference: instrumentation. */
int glide_alg_bytes(glide_handle h, double* bytes);
/* One launch of the linear smoother's block factorisation (part 0) or of its
 * block sweep x -= omega B^-1 r over the current residual (part 1), on the
 * tangent system (adjoint = 0) or the adjoint system (adjoint = 1) of
 * `level`, nothing before or after it: for timing the two kernels alone.  A
 * sweep without a preceding factorisation of the same state reads whatever
 * the factor buffers hold.  No counterpart in the reference:
 * instrumentation. */
int glide_block_smoother_part(glide_handle h, int level, double dt, int adjoint, int part, void* stream);
/* Kernel tuning knobs (no counterpart in the reference).
 * GLIDE_TUNE_SWEEP_BLOCKS_PER_SM: 1 or 2 resident Vanka-sweep blocks per SM.
 * GLIDE_TUNE_MIXED_INNER_VCYCLES: binary32 V-cycles per defect correction
 * of a GLIDE_MIXED handle (default 1). */
#define GLIDE_TUNE_SWEEP_BLOCKS_PER_SM 1
#define GLIDE_TUNE_MIXED_INNER_VCYCLES 2
/* GLIDE_TUNE_FORWARD_METHOD: 0 = FASCD V-cycles only (the reference's
 * method); 1 = FASCD until the relative residual reaches 10^-k
 * (GLIDE_TUNE_NEWTON_SWITCH_EXP10 = k, default 2), then Newton steps whose
 * correction is solved by GLIDE_TUNE_TANGENT_VCYCLES V-cycles (default 1) of
 * the tangent linear multigrid (schedule and smoother: config selector 2).
 * GLIDE_MIXED handles default to 1. */
#define GLIDE_TUNE_FORWARD_METHOD 3
#define GLIDE_TUNE_NEWTON_SWITCH_EXP10 4
#define GLIDE_TUNE_TANGENT_VCYCLES 5
/* GLIDE_TUNE_TMA_STAGING: 1 (default) stages the halo tiles of the stencil
 * kernels with TMA bulk tensor copies on levels at least 24 x 20 cells;
 * 0 uses clamped per-thread loads everywhere (same results). */
#define GLIDE_TUNE_TMA_STAGING 6
/* GLIDE_TUNE_REPORT_NOT_CONVERGED: 1 makes glide_forward / glide_backward
 * return GLIDE_ERR_NOT_CONVERGED when the solve ends short of its
 * tolerances; 0 (default) returns GLIDE_OK as the reference would. */
#define GLIDE_TUNE_REPORT_NOT_CONVERGED 7
/* GLIDE_TUNE_TMA_GIVE_UP: a stencil block's first wait for its staged tile
 * copies polls at most 2^22 times, then gives up, sets the handle's error
 * word and returns; the call fails with GLIDE_ERR_TIMEOUT at its next norm
 * read, and the word is cleared when reported.  1 makes that first wait give
 * up at once, which tests the path (the block still waits, bounded, for its
 * copies to land before it returns); 0 restores the default. */
#define GLIDE_TUNE_TMA_GIVE_UP 8
int glide_set_tuning(glide_handle h, int key, int value);

int glide_set_rhs(glide_handle h, int level, double dt, void* stream);
int glide_compute_phi(glide_handle h, int level, double relaxation, void* stream);
int glide_residual(glide_handle h, int level, double dt, int flags, double* norms3, void* stream);
int glide_vanka_sweep(glide_handle h, int level, double dt, int n, int flags, int* newton_iters,
                      void* stream);
/* Local 5x5 Vanka systems of every cell of a level at its current state
 * (ForwardOperators.vanka_dump, glide/operators.py:253-273, glide/cuda/vanka.cu:801-908):
 * J (ny*nx x 25, row-major per cell) and r (ny*nx x 5), device arrays of the
 * handle's value type (binary64 for GLIDE_F64 and GLIDE_MIXED). */
int glide_vanka_dump(glide_handle h, int level, double dt, void* J, void* r, void* stream);
int glide_forward(glide_handle h, double dt, int start_level, glide_stats* stats, void* stream);

int glide_adjoint_residual(glide_handle h, int level, double dt, double* norms3, void* stream);
int glide_vjp(glide_handle h, int level, double dt, void* stream);
/* JVP_* = J(x) VAR_* at the level's state with the grounded fraction held
 * fixed.  reference_rows = 1 follows ForwardOperators.compute_jvp
 * (glide/operators.py:129-171, glide/cuda/residuals.cu:341-660): zero on the
 * Dirichlet faces, (1 - mask) times the mass rows.  reference_rows = 0 gives
 * the Jacobian the Newton iteration uses (identity rows there).  flags are
 * the reference's keyword arguments: GLIDE_USE_MASK (use_mask=True, its
 * default; without it the mask reads as 0) and GLIDE_FREEZE_CALVING
 * (freeze_calving=True: calving rate 0).  Any other flag is GLIDE_ERR_ARG. */
int glide_jvp(glide_handle h, int level, double dt, int reference_rows, int flags, void* stream);
int glide_adjoint_sweep(glide_handle h, int level, double dt, int n, void* stream);
int glide_gradients(glide_handle h, int level, double dt, int grad_mask, void* stream);
int glide_backward(glide_handle h, double dt, int start_level, int grad_mask, glide_stats* stats,
                   void* stream);
/* One V-cycle from `level` and nothing around it: FASCDSolver.vcycle
 * (glide/multigrid.py:536-645) for which = 0, FASAdjointSolver.vcycle
 * (glide/multigrid.py:905-973) for which = 1.  finest != 0 takes the
 * top-of-cycle snapshot (w = x, chi = thklim - H) as the reference's
 * finest=True does.  The right-hand side of `level` must already be set
 * (glide_set_rhs for the forward system, the adjoint right-hand side for the
 * adjoint); no residual is evaluated.  Runs the handle's binary64 hierarchy on
 * a mixed handle. */
int glide_vcycle(glide_handle h, int which, int level, int finest, double dt, void* stream);

/* Residual and its norms on caller-owned device arrays, allocating nothing.
 * No counterpart in the reference.  It computes what glide_residual computes
 * for one level, for hosts that may not allocate device memory after start-up
 * and so cannot create a handle.  All arrays are binary64 device memory, row-major with leading
 * dimensions ld_u (u, f_u, r_u: ny x (nx+1)), ld_v (v, f_v, r_v: (ny+1) x nx)
 * and ld_c (cell arrays: ny x nx).  Unless flags has GLIDE_FREEZE_PHI, phi is
 * first recomputed from H and bed (it is in/out, and must hold finite values
 * on entry: the zero-weight blend with its old values still reads them).  Flags GLIDE_USE_MASK,
 * GLIDE_OPERATOR_ONLY (f_* may then be NULL) and GLIDE_FREEZE_CALVING act as
 * in glide_residual.  norms (device, 4 doubles) receives |r_u|, |r_v|, |r_H|
 * and the combined norm; it is written on `stream`, not synchronised.
 * Limits: at most 65,536 tiles of 16 x 16 cells (4096 x 4096 cells, for
 * example) and at most 65,535 rows; larger grids return GLIDE_ERR_SHAPE.  The
 * scratch is one static device array per GPU (1.5 MiB).  Every call looks up
 * its address in the current context; the first call in a context also loads
 * the module that holds it, so make that call before any stream capture.
 * Nothing needs zeroing beforehand.
 * Calls that overlap in time on one GPU share that scratch and race. */
int glide_residual_norms_noalloc(int ny, int nx, double dx, double dt, const glide_phys* phys,
                                 const double* u, int ld_u, const double* v, int ld_v, const double* H,
                                 double* phi, const double* mask, const double* f_u, const double* f_v,
                                 const double* f_H, const double* bed, const double* B, const double* beta,
                                 const double* gamma, int ld_c, int flags, double* r_u, double* r_v,
                                 double* r_H, double* norms, void* stream);
/* Message of the last failed glide_residual_norms_noalloc on this thread. */
const char* glide_noalloc_last_error(void);

/* One restriction or prolongation of one field between caller arrays, no
 * handle needed: the reference's Multigrid.restrict_vfacet / restrict_hfacet /
 * restrict_cell / prolongate_vfacet / prolongate_hfacet / prolongate_cell
 * (glide/multigrid.py:119-259) over the kernels of glide/cuda/transfer.cu.
 * ny_fine, nx_fine: the fine grid's cell counts (even); the coarse grid has
 * half of each.  Array shapes, rows x cols, fine / coarse:
 *   VFACET  (u faces)  ny_fine x (nx_fine+1)  /  ny_c x (nx_c+1)
 *   HFACET  (v faces)  (ny_fine+1) x nx_fine  /  (ny_c+1) x nx_c
 *   CELL               ny_fine x nx_fine      /  ny_c x nx_c
 * A restriction reads the fine array (src) and writes the coarse one (dst);
 * a prolongation the other way round.  ld_src / ld_dst are leading
 * dimensions in elements; src and dst must not overlap.  dtype GLIDE_F64 or
 * GLIDE_F32.  GLIDE_PROLONG_HFACET_AS_VFACET_* is what the reference's
 * prolongate_hfacet runs: the u-face kernels over the flat memory of v-face
 * arrays (square grids only, else GLIDE_ERR_SHAPE).  Asynchronous on
 * `stream`; errors in glide_last_error(). */
#define GLIDE_RESTRICT_VFACET 0
#define GLIDE_RESTRICT_HFACET 1
#define GLIDE_RESTRICT_CELL_AVG 2
#define GLIDE_RESTRICT_CELL_MAX 3
#define GLIDE_RESTRICT_CELL_MIN 4
#define GLIDE_RESTRICT_CELL_VAR 5
#define GLIDE_PROLONG_VFACET_INJECTION 6
#define GLIDE_PROLONG_VFACET_BILINEAR 7
#define GLIDE_PROLONG_HFACET_INJECTION 8
#define GLIDE_PROLONG_HFACET_BILINEAR 9
#define GLIDE_PROLONG_CELL_INJECTION 10
#define GLIDE_PROLONG_CELL_BILINEAR 11
#define GLIDE_PROLONG_HFACET_AS_VFACET_INJECTION 12
#define GLIDE_PROLONG_HFACET_AS_VFACET_BILINEAR 13
int glide_transfer(int op, int dtype, int ny_fine, int nx_fine, const void* src, int ld_src, void* dst, int ld_dst,
                   void* stream);

/* Groups: one solve of many handles in grouped launches.  No counterpart in
 * the reference, whose models solve one grid at a time (IceDynamics.forward /
 * backward, glide/model.py:62-94); each member is an ordinary handle and
 * keeps that API.  A group solve runs every member's cycle -- the same
 * launches, in the same order, with the same arguments as glide_forward /
 * glide_backward on that member -- but issues each kind of launch once for
 * all members: blocks map to (member, tile) through a table in the launch's
 * parameters.  The cycle of all members is one CUDA graph, and each member's
 * convergence test (its own tolerances and cycle cap) runs on the device, so
 * a converged member's launches are skipped from the next cycle on.  Results
 * equal the members' own solves.
 *
 * Members: handles of one dtype, GLIDE_F64 or GLIDE_F32 (mixed-precision
 * handles: GLIDE_ERR_STATE), each at most once; they must outlive the group
 * and must not be used from another thread while a group call runs.  Each
 * member solves with its own schedule, tolerances and forward method: the
 * guarded Newton steps' decisions (when to step, undoing a step whose
 * residual grew, falling back to FASCD) are taken on the device as
 * glide_forward takes them on the host.  stats: n entries, one per member
 * (may be NULL).  A
 * member whose residual becomes non-finite returns GLIDE_ERR_NONFINITE after
 * the others finish; one whose staged tiles fail (a bounded wait that gave
 * up: GLIDE_ERR_TIMEOUT; staging maps in device memory that fail their
 * check, so that no copy used them: GLIDE_ERR_STATE) stops and is reported
 * the same way.  The staging maps of a plan are copied to the device on the
 * call's stream before its graph is captured.  Plans (the merged launch lists and their graphs) are
 * rebuilt when dt, start_level, grad_mask or any member's configuration
 * changes. */
typedef struct glide_group_s* glide_group;
int glide_group_create(const glide_handle* members, int n, glide_group* out);
int glide_group_destroy(glide_group g);
int glide_group_forward(glide_group g, double dt, int start_level, glide_stats* stats, void* stream);
int glide_group_backward(glide_group g, double dt, int start_level, int grad_mask, glide_stats* stats,
                         void* stream);
/* Launch shape of the grouped launches (no counterpart in the reference).
 * GLIDE_GROUP_TUNE_WAVES: 0 (default) launches one block per tile of every
 * member; value > 0 makes the grid value x the resident blocks of the GPU,
 * every block striding over the tiles.  Plans are recaptured on the next
 * call. */
#define GLIDE_GROUP_TUNE_WAVES 1
/* GLIDE_GROUP_TUNE_SPOIL_MAPS: 1 uploads every staging map without the tag
 * the kernels check before their first copy, which tests that check: each
 * member stops after its first stencil launch and the call fails with
 * GLIDE_ERR_STATE, no copy having used the maps; 0 (default) restores the
 * plain upload.  Plans are rebuilt on the next call. */
#define GLIDE_GROUP_TUNE_SPOIL_MAPS 2
int glide_group_set_tuning(glide_group g, int key, int value);
/* launches: grouped launches issued so far.  shape (4 ints, may be NULL): the
 * last forward cycle's grouped launches and the members' launches they
 * carry, then the same for the adjoint cycle. */
int glide_group_counters(glide_group g, long long* launches, int* shape);

#ifdef __cplusplus
}
#endif
#endif /* GLIDE_B200_H */
