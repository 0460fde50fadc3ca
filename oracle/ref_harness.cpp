// ref_harness.cpp -- host build of the reference's own CUDA kernels (test
// infrastructure; never shipped, never timed as the product).
//
// The reference kernel files (glide/cuda/*.cu of JacobDowns/glide) are
// #included unmodified from the reference checkout given on the command line
// (-I<reference>/glide/cuda) and executed on host cores through simt_host.hpp.
// Output goes only to oracle/_ref/.  Two builds exist:
//   GLIDE_REF_FP64 undefined: the kernels as written (binary32 arithmetic,
//                            correctly rounded host math instead of fast-math)
//   GLIDE_REF_FP64 defined  : every `float` of the reference source becomes
//                            `double` (float literals such as 0.917f keep their
//                            binary32 value), giving the binary64 evaluation of
//                            the same discrete operator.
// Each exported gref_* function launches one kernel with the grid/block the
// caller passes, exactly like cupy.RawModule's kernel(grid, block, args).
#include "simt_host.hpp"

#ifdef GLIDE_REF_FP64
#define fmaxf fmax
#define fminf fmin
#define sqrtf sqrt
#define fabsf fabs
#define copysignf copysign
#define float double
#endif

#include "common.cu"
#include "viscosity.cu"
#include "stress.cu"
#include "flux.cu"
#include "residuals.cu"
#include "vanka.cu"
#include "grad.cu"
#include "transfer.cu"
// The enthalpy module is compiled by the reference with its physical constants
// injected as #define lines (glide/enthalpy.py:229-246); build_oracle.py writes
// the same lines into oracle/_ref/enthalpy_defines.h.
#include "enthalpy_defines.h"
#include "enthalpy.cu"

#ifdef GLIDE_REF_FP64
#undef float
typedef double ref_real;
#else
typedef float ref_real;
#endif

namespace {
inline simt::uint3_ d3(int x, int y, int z) { return simt::uint3_{unsigned(x), unsigned(y), unsigned(z)}; }
}

#define GREF_PHYS_PARAMS                                                          \
    ref_real n, ref_real eps_reg, ref_real flotation_reg_driving, ref_real m,     \
        ref_real u_reg, ref_real water_drag, ref_real flotation_reg_sliding,      \
        ref_real calving_rate, ref_real flotation_reg_calving, ref_real dx,       \
        ref_real dt
#define GREF_PHYS_ARGS                                                            \
    n, eps_reg, flotation_reg_driving, m, u_reg, water_drag,                      \
        flotation_reg_sliding, calving_rate, flotation_reg_calving, dx, dt

extern "C" {

int gref_real_bytes() { return int(sizeof(ref_real)); }

void gref_compute_residual(int gx, int gy, int bx, int by,
                           ref_real* r_u, ref_real* r_v, ref_real* r_H,
                           const ref_real* u, const ref_real* v, const ref_real* H,
                           const ref_real* phi, const ref_real* mask,
                           const ref_real* f_u, const ref_real* f_v, const ref_real* f_H,
                           const ref_real* bed, const ref_real* B, const ref_real* beta,
                           const ref_real* gamma, bool use_forcing, bool use_mask,
                           GREF_PHYS_PARAMS, int ny, int nx, int stride, int halo) {
    simt::launch(d3(gx, gy, 1), d3(bx, by, 1), [&] {
        compute_residual(r_u, r_v, r_H, u, v, H, phi, mask, f_u, f_v, f_H, bed, B, beta,
                         gamma, use_forcing, use_mask, GREF_PHYS_ARGS, ny, nx, stride, halo);
    });
}

void gref_compute_jvp(int gx, int gy, int bx, int by,
                      ref_real* jvp_u, ref_real* jvp_v, ref_real* jvp_H,
                      const ref_real* u, const ref_real* v, const ref_real* H,
                      const ref_real* d_u, const ref_real* d_v, const ref_real* d_H,
                      const ref_real* phi, const ref_real* mask,
                      const ref_real* f_u, const ref_real* f_v, const ref_real* f_H,
                      const ref_real* bed, const ref_real* B, const ref_real* beta,
                      const ref_real* gamma, bool use_mask,
                      GREF_PHYS_PARAMS, int ny, int nx, int stride, int halo) {
    simt::launch(d3(gx, gy, 1), d3(bx, by, 1), [&] {
        compute_jvp(jvp_u, jvp_v, jvp_H, u, v, H, d_u, d_v, d_H, phi, mask, f_u, f_v, f_H,
                    bed, B, beta, gamma, use_mask, GREF_PHYS_ARGS, ny, nx, stride, halo);
    });
}

void gref_compute_vjp(int gx, int gy, int bx, int by,
                      ref_real* vjp_u, ref_real* vjp_v, ref_real* vjp_H,
                      const ref_real* u, const ref_real* v, const ref_real* H,
                      const ref_real* l_u, const ref_real* l_v, const ref_real* l_H,
                      const ref_real* phi, const ref_real* mask,
                      const ref_real* f_u, const ref_real* f_v, const ref_real* f_H,
                      const ref_real* bed, const ref_real* B, const ref_real* beta,
                      const ref_real* gamma, bool use_forcing, bool use_mask,
                      GREF_PHYS_PARAMS, int ny, int nx, int stride, int halo) {
    simt::launch(d3(gx, gy, 1), d3(bx, by, 1), [&] {
        compute_vjp(vjp_u, vjp_v, vjp_H, u, v, H, l_u, l_v, l_H, phi, mask, f_u, f_v, f_H,
                    bed, B, beta, gamma, use_forcing, use_mask, GREF_PHYS_ARGS, ny, nx,
                    stride, halo);
    });
}

void gref_compute_grounded(int gx, int gy, int bx, int by, ref_real* grounded,
                           const ref_real* H, const ref_real* bed, ref_real sigmoid_c,
                           ref_real relaxation, int ny, int nx, int stride, int halo) {
    simt::launch(d3(gx, gy, 1), d3(bx, by, 1), [&] {
        compute_grounded(grounded, H, bed, sigmoid_c, relaxation, ny, nx, stride, halo);
    });
}

void gref_vanka_smooth(int gx, int gy, int bx, int by,
                       ref_real* delta_u, ref_real* delta_v, ref_real* delta_H, ref_real* mask,
                       const ref_real* u, const ref_real* v, const ref_real* H,
                       const ref_real* phi, const ref_real* f_u, const ref_real* f_v,
                       const ref_real* f_H, const ref_real* bed, const ref_real* B,
                       const ref_real* beta, const ref_real* gamma, GREF_PHYS_PARAMS,
                       int ny, int nx, int stride, int halo, int newton_steps,
                       ref_real relaxation, ref_real ssa_damping, ref_real mc_damping) {
    simt::launch(d3(gx, gy, 1), d3(bx, by, 1), [&] {
        vanka_smooth(delta_u, delta_v, delta_H, mask, u, v, H, phi, f_u, f_v, f_H, bed, B,
                     beta, gamma, GREF_PHYS_ARGS, ny, nx, stride, halo, newton_steps,
                     relaxation, ssa_damping, mc_damping);
    });
}

void gref_vanka_smooth_adjoint(int gx, int gy, int bx, int by,
                               ref_real* l_u_out, ref_real* l_v_out, ref_real* l_H_out,
                               const ref_real* u, const ref_real* v, const ref_real* H,
                               const ref_real* phi, const ref_real* mask,
                               const ref_real* r_u, const ref_real* r_v, const ref_real* r_H,
                               const ref_real* bed, const ref_real* B, const ref_real* beta,
                               const ref_real* gamma, GREF_PHYS_PARAMS, int ny, int nx,
                               int stride, int halo, ref_real ssa_damping,
                               ref_real mc_damping) {
    simt::launch(d3(gx, gy, 1), d3(bx, by, 1), [&] {
        vanka_smooth_adjoint(l_u_out, l_v_out, l_H_out, u, v, H, phi, mask, r_u, r_v, r_H,
                             bed, B, beta, gamma, GREF_PHYS_ARGS, ny, nx, stride, halo,
                             ssa_damping, mc_damping);
    });
}

void gref_vanka_dump(int gx, int gy, int bx, int by, ref_real* J_array, ref_real* r_array,
                     const ref_real* u, const ref_real* v, const ref_real* H,
                     const ref_real* phi, const ref_real* f_u, const ref_real* f_v,
                     const ref_real* f_H, const ref_real* bed, const ref_real* B,
                     const ref_real* beta, const ref_real* gamma, GREF_PHYS_PARAMS,
                     int ny, int nx, int stride, int halo) {
    simt::launch(d3(gx, gy, 1), d3(bx, by, 1), [&] {
        vanka_dump(J_array, r_array, u, v, H, phi, f_u, f_v, f_H, bed, B, beta, gamma,
                   GREF_PHYS_ARGS, ny, nx, stride, halo);
    });
}

#define GREF_GRAD(NAME)                                                                 \
    void gref_##NAME(int gx, int gy, int bx, int by, ref_real* grad,                    \
                     const ref_real* u, const ref_real* v, const ref_real* H,           \
                     const ref_real* l_u, const ref_real* l_v, const ref_real* l_H,     \
                     const ref_real* phi, const ref_real* mask, const ref_real* bed,    \
                     const ref_real* B, const ref_real* beta, const ref_real* gamma,    \
                     GREF_PHYS_PARAMS, int ny, int nx, int stride, int halo) {          \
        simt::launch(d3(gx, gy, 1), d3(bx, by, 1), [&] {                                \
            NAME(grad, u, v, H, l_u, l_v, l_H, phi, mask, bed, B, beta, gamma,          \
                 GREF_PHYS_ARGS, ny, nx, stride, halo);                                 \
        });                                                                             \
    }
GREF_GRAD(compute_gradient_beta)
GREF_GRAD(compute_gradient_bed)

#define GREF_TRANSFER(NAME)                                                             \
    void gref_##NAME(int gx, int bx, const ref_real* src, ref_real* dst, int a, int b) { \
        simt::launch(d3(gx, 1, 1), d3(bx, 1, 1), [&] { NAME(src, dst, a, b); });        \
    }
GREF_TRANSFER(restrict_vfacet)
GREF_TRANSFER(restrict_hfacet)
GREF_TRANSFER(restrict_cell_avg)
GREF_TRANSFER(restrict_cell_max)
GREF_TRANSFER(restrict_cell_min)
GREF_TRANSFER(restrict_cell_var)
GREF_TRANSFER(prolongate_vfacet_injection)
GREF_TRANSFER(prolongate_vfacet_bilinear)
GREF_TRANSFER(prolongate_hfacet_injection)
GREF_TRANSFER(prolongate_hfacet_bilinear)
GREF_TRANSFER(prolongate_cell_injection)
GREF_TRANSFER(prolongate_cell_bilinear)

#define GREF_ENTHALPY_ARRAYS                                                          \
    const ref_real *E, const ref_real *E_prev, const ref_real *f_E, const ref_real *u3d,  \
        const ref_real *v3d, const ref_real *omega, const ref_real *H,                    \
        const ref_real *H_prev, const ref_real *E_surface, ref_real dx, ref_real dt,      \
        ref_real drain_rate, ref_real h_thin, ref_real lf_c, int term_flags

void gref_enthalpy_compute_residual(int gx, int bx, ref_real* out, GREF_ENTHALPY_ARRAYS,
                                    int use_forcing, int ny, int nx, int nz) {
    simt::launch(d3(gx, 1, 1), d3(bx, 1, 1), [&] {
        enthalpy_compute_residual(out, E, E_prev, f_E, u3d, v3d, omega, H, H_prev, E_surface, dx, dt,
                                  drain_rate, h_thin, lf_c, term_flags, use_forcing, ny, nx, nz);
    });
}

void gref_enthalpy_column_smooth(int gx, int bx, ref_real* delta_E, GREF_ENTHALPY_ARRAYS, int ny,
                                 int nx, int nz, int n_newton, ref_real relaxation) {
    simt::launch(d3(gx, 1, 1), d3(bx, 1, 1), [&] {
        enthalpy_column_smooth(delta_E, E, E_prev, f_E, u3d, v3d, omega, H, H_prev, E_surface, dx, dt,
                               drain_rate, h_thin, lf_c, term_flags, ny, nx, nz, n_newton, relaxation);
    });
}

void gref_enthalpy_layer_smooth(int gx, int bx, ref_real* delta_E, GREF_ENTHALPY_ARRAYS, int ny,
                                int nx, int nz) {
    simt::launch(d3(gx, 1, 1), d3(bx, 1, 1), [&] {
        enthalpy_layer_smooth(delta_E, E, E_prev, f_E, u3d, v3d, omega, H, H_prev, E_surface, dx, dt,
                              drain_rate, h_thin, lf_c, term_flags, ny, nx, nz);
    });
}

void gref_compute_omega(int gx, int bx, ref_real* omega, const ref_real* u3d, const ref_real* v3d,
                        const ref_real* H, const ref_real* dh_dt, const ref_real* bmb, ref_real dx, int ny,
                        int nx, int nz) {
    simt::launch(d3(gx, 1, 1), d3(bx, 1, 1), [&] {
        compute_omega(omega, u3d, v3d, H, dh_dt, bmb, dx, ny, nx, nz);
    });
}

}  // extern "C"
