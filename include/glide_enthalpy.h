/* glide_enthalpy.h -- C ABI of the B200-native enthalpy column solver
 * (drop-in for glide/enthalpy.py EnthalpyOperators and the device work of
 * glide/model.py ThermalModel.step, JacobDowns/glide).  Binary64 throughout.
 *
 * Conventions as in glide_b200.h: device pointers, `stream` a cudaStream_t
 * passed as void*, every call returns GLIDE_OK (0) or a GLIDE_ERR_* code and
 * glide_enthalpy_last_error() gives the message.  A handle is not
 * thread-safe.
 *
 * Layout: the handle owns its 3-D node arrays layer-major, node (k, i, j)
 * at k*ny*nx + i*nx + j (the reference stores them (ny, nx, nz), k fastest;
 * a (ny, nx, nz)-shaped view with strides (nx, 1, ny*nx) reads the same
 * memory).  u3d is (nz, ny, nx+1) and v3d (nz, ny+1, nx), as in the
 * reference.  2-D arrays are (ny, nx) row-major.
 *
 * Reference interfaces each entry point replaces:
 *   glide_enthalpy_create / destroy     EnthalpyOperators.__init__ (glide/enthalpy.py:220-280)
 *   glide_enthalpy_field_ptr            EnthalpyState / EnthalpyForcing / EnthalpyVelocity arrays,
 *                                       r_E, f_E, delta_E, H_prev (glide/enthalpy.py:96-158, :248-277)
 *   glide_enthalpy_set_config           ColumnSmootherConfig, EnthalpyTermFlags, drain_rate, h_thin
 *                                       (glide/enthalpy.py:108-203)
 *   glide_enthalpy_set_inputs           grid.state.H and the velocity the kernels read
 *                                       (broadcast_velocity, glide/enthalpy.py:289-301)
 *   glide_enthalpy_snapshot             E_prev <- E, H_prev <- H (set_rhs(snapshot=True),
 *                                       ThermalModel.pre_momentum, glide/model.py:155-164)
 *   glide_enthalpy_set_rhs              EnthalpyOperators.set_rhs (glide/enthalpy.py:473-519)
 *   glide_enthalpy_residual             EnthalpyOperators.compute_residual (glide/enthalpy.py:341-364)
 *   glide_enthalpy_column_smooth        EnthalpyOperators.column_smooth (glide/enthalpy.py:366-393)
 *   glide_enthalpy_layer_smooth         EnthalpyOperators.layer_smooth (glide/enthalpy.py:395-424)
 *   glide_enthalpy_column_sweep         EnthalpyOperators.column_sweep (glide/enthalpy.py:426-471)
 *   glide_enthalpy_compute_omega        EnthalpyOperators.compute_omega (glide/enthalpy.py:303-339) and
 *                                       ThermalModel._compute_omega (glide/model.py:237-258)
 *   glide_enthalpy_frictional_heating   ThermalModel._compute_frictional_heating (glide/model.py:224-235)
 *   glide_enthalpy_arrhenius            EnthalpyOperators.get_arrhenius_factor (glide/enthalpy.py:600-643)
 *                                       with ThermalModel's B feedback (glide/model.py:212-222)
 */
#ifndef GLIDE_ENTHALPY_H
#define GLIDE_ENTHALPY_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct glide_enthalpy* glide_enthalpy_handle;

/* Arrays owned by the handle.  3-D: layer-major (see above). */
enum glide_enthalpy_field {
    GLIDE_ENTH_E = 0,       /* (nz, ny, nx)   scaled enthalpy E / E_SCALE */
    GLIDE_ENTH_E_PREV,      /* (nz, ny, nx) */
    GLIDE_ENTH_F_E,         /* (nz, ny, nx)   precomputed forcing */
    GLIDE_ENTH_OMEGA,       /* (nz, ny, nx)   omega = H sigma_dot, m/s */
    GLIDE_ENTH_R_E,         /* (nz, ny, nx)   residual */
    GLIDE_ENTH_DELTA_E,     /* (nz, ny, nx)   smoother correction */
    GLIDE_ENTH_PHI_STRAIN,  /* (nz, ny, nx)   strain heating, W m^-3 */
    GLIDE_ENTH_U3D,         /* (nz, ny, nx+1) layer x-velocity, m/s */
    GLIDE_ENTH_V3D,         /* (nz, ny+1, nx) layer y-velocity, m/s */
    GLIDE_ENTH_H_PREV,      /* (ny, nx)       thickness at the previous step */
    GLIDE_ENTH_E_SURFACE,   /* (ny, nx)       surface Dirichlet value */
    GLIDE_ENTH_Q_GEO,       /* (ny, nx)       geothermal flux, W m^-2 */
    GLIDE_ENTH_Q_FH,        /* (ny, nx)       frictional heating, W m^-2 */
    GLIDE_ENTH_N_FIELDS
};

/* Term flags (EnthalpyTermFlags.bitmask) */
#define GLIDE_ENTH_HORIZ_ADV 1
#define GLIDE_ENTH_SIGMA_DOT 2
#define GLIDE_ENTH_DRAINAGE 4

typedef struct {
    double omega;               /* smoother update weight (1.0) */
    int n_newton;               /* Newton steps per column smooth (3) */
    double relaxation;          /* Newton step length (1.0) */
    double relative_tolerance;  /* column_sweep stop (1e-5) */
    double absolute_tolerance;  /* column_sweep stop (1e-2) */
    double lf_c;                /* Lax-Friedrichs regulariser (1e-12) */
    double drain_rate;          /* s^-1 (0.01 a^-1) */
    double h_thin;              /* m (25) */
    int term_flags;             /* GLIDE_ENTH_* (7) */
} glide_enthalpy_config;

/* What the kernels read besides the handle's own arrays.  H (ny, nx) with
 * leading dimension ld_H.  Velocity at layer k, row i, column j:
 * u[k*u_layer + i*ld_u + j]; u_layer = 0 reads one 2-D field for every
 * layer.  All velocity reads are divided by vel_div.  NULL u / v select the
 * handle's own U3D / V3D. */
typedef struct {
    const double* H;
    int ld_H;
    const double* u;
    int ld_u;
    long long u_layer;
    const double* v;
    int ld_v;
    long long v_layer;
    double vel_div;
} glide_enthalpy_inputs;

#define GLIDE_ENTH_MAX_HISTORY 256
typedef struct {
    int iterations;      /* sweeps run */
    double initial_norm; /* max |r_E| before the sweep */
    double final_norm;
    double history[GLIDE_ENTH_MAX_HISTORY]; /* max |r_E| after each sweep */
} glide_enthalpy_stats;

const char* glide_enthalpy_last_error(void);

/* 2 <= nz <= 64; dx in m. */
int glide_enthalpy_create(int ny, int nx, int nz, double dx, glide_enthalpy_handle* out);
int glide_enthalpy_destroy(glide_enthalpy_handle h);
int glide_enthalpy_field_ptr(glide_enthalpy_handle h, int field, void** ptr);
int glide_enthalpy_set_config(glide_enthalpy_handle h, const glide_enthalpy_config* c);
int glide_enthalpy_get_config(glide_enthalpy_handle h, glide_enthalpy_config* c);
int glide_enthalpy_set_inputs(glide_enthalpy_handle h, const glide_enthalpy_inputs* in);
/* Launch shapes, no counterpart in the reference: resident blocks per SM the
 * residual / layer kernels (3 to 6; default 3) and the column kernel (2 to
 * 6; default 4) are compiled for, and whether the column kernel prefers the
 * largest L1 (value 1) for its per-column Thomas arrays. */
#define GLIDE_ENTH_TUNE_POINT_BLOCKS 1
#define GLIDE_ENTH_TUNE_COLUMN_BLOCKS 2
#define GLIDE_ENTH_TUNE_COLUMN_L1 3
/* GLIDE_ENTH_TUNE_COLUMN_KERNEL: 1 (default) runs the column smoother with one
 * Thomas factor in shared memory, the other and the iterate in L2-resident
 * arrays, sized for 6 resident blocks of 64 threads per SM; 2 the same sized
 * for 8 (fewer registers per thread); 0 the one-thread-per-column kernel with
 * per-thread arrays.  Results agree to rounding. */
#define GLIDE_ENTH_TUNE_COLUMN_KERNEL 4
int glide_enthalpy_set_tuning(glide_enthalpy_handle h, int key, int value);
int glide_enthalpy_snapshot(glide_enthalpy_handle h, void* stream);
int glide_enthalpy_set_rhs(glide_enthalpy_handle h, void* stream);
/* max_abs (host, may be NULL) receives max |r_E| and synchronises `stream`. */
int glide_enthalpy_residual(glide_enthalpy_handle h, double dt, int use_forcing, double* max_abs,
                            void* stream);
int glide_enthalpy_column_smooth(glide_enthalpy_handle h, double dt, void* stream);
int glide_enthalpy_layer_smooth(glide_enthalpy_handle h, double dt, void* stream);
/* Up to n_iter sweeps (column smooth, E += omega delta, then when
 * `alternating` layer smooth, E += omega delta), stopping after the first
 * sweep whose max |r_E| is below relative_tolerance * initial or
 * absolute_tolerance.  The stop test runs on the device; the call
 * synchronises `stream` once, at the end. */
int glide_enthalpy_column_sweep(glide_enthalpy_handle h, double dt, int n_iter, int alternating,
                                glide_enthalpy_stats* stats, void* stream);
/* dh_dt (ny, nx, leading dimension ld_dh) in the velocity's units, or NULL for
 * (H - H_PREV) / dh_div; bmb NULL for zero.  The velocity is read without
 * vel_div; omega is divided by omega_div. */
int glide_enthalpy_compute_omega(glide_enthalpy_handle h, const double* dh_dt, int ld_dh, const double* bmb,
                                 int ld_bmb, double dh_div, double omega_div, void* stream);
/* Q_FH = beta |u_b|^(m+1) from layer 0 of the velocity (divided by vel_div). */
int glide_enthalpy_frictional_heating(glide_enthalpy_handle h, const double* beta, int ld_beta, double m,
                                      double u_reg, void* stream);
/* B (ny, nx, leading dimension ld_B) = mean_k(A(T, water))^(-1/n_glen) / scale. */
int glide_enthalpy_arrhenius(glide_enthalpy_handle h, double n_glen, double scale, double* B, int ld_B,
                             void* stream);
/* Kernels this handle has launched so far, and their algorithmic bytes (the
 * binary64 values each must read and write once; column-sweep passes skipped
 * by the stop test count as launches but move no bytes).  Either pointer may
 * be NULL.  No counterpart in the reference: instrumentation. */
int glide_enthalpy_counters(glide_enthalpy_handle h, long long* launches, double* alg_bytes);

#ifdef __cplusplus
}
#endif
#endif /* GLIDE_ENTHALPY_H */
