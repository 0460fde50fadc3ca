// ref_gpu.cu -- the reference's own CUDA kernels built for sm_100a (test
// infrastructure: a baseline that is timed beside the product, never the
// product).
//
// The kernel files of JacobDowns/glide (glide/cuda/*.cu) are #included
// unmodified from the reference checkout named on the command line
// (-I<reference>/glide/cuda), in the order the reference concatenates its
// forward module (glide/operators.py:20-22), followed by its transfer module
// (glide/multigrid.py), and compiled with --use_fast_math as the reference's
// cupy.RawModule compiles them.  Output goes only to oracle/_ref/.
//
// Each exported grg_* function launches one kernel with the grid and block
// the caller passes, on the caller's stream, exactly as cupy.RawModule's
// kernel(grid, block, args) does, and returns the launch's error code.
#include <cuda_runtime.h>

#include "common.cu"
#include "viscosity.cu"
#include "stress.cu"
#include "flux.cu"
#include "residuals.cu"
#include "vanka.cu"
#include "grad.cu"
#include "transfer.cu"

#define GRG_PHYS_PARAMS                                                                            \
    float n, float eps_reg, float flotation_reg_driving, float m, float u_reg, float water_drag,  \
        float flotation_reg_sliding, float calving_rate, float flotation_reg_calving, float dx, float dt
#define GRG_PHYS_ARGS \
    n, eps_reg, flotation_reg_driving, m, u_reg, water_drag, flotation_reg_sliding, calving_rate, \
        flotation_reg_calving, dx, dt

static dim3 d2(int x, int y) { return dim3(unsigned(x), unsigned(y), 1u); }
static cudaStream_t st(void* s) { return static_cast<cudaStream_t>(s); }

extern "C" {

int grg_compute_grounded(int gx, int gy, int bx, int by, float* phi, const float* H, const float* bed,
                         float sigmoid_c, float relaxation, int ny, int nx, int stride, int halo, void* s) {
    compute_grounded<<<d2(gx, gy), d2(bx, by), 0, st(s)>>>(phi, H, bed, sigmoid_c, relaxation, ny, nx, stride,
                                                           halo);
    return int(cudaGetLastError());
}

int grg_compute_residual(int gx, int gy, int bx, int by, float* r_u, float* r_v, float* r_H, const float* u,
                         const float* v, const float* H, const float* phi, const float* mask, const float* f_u,
                         const float* f_v, const float* f_H, const float* bed, const float* B, const float* beta,
                         const float* gamma, int use_forcing, int use_mask, GRG_PHYS_PARAMS, int ny, int nx,
                         int stride, int halo, void* s) {
    compute_residual<<<d2(gx, gy), d2(bx, by), 0, st(s)>>>(r_u, r_v, r_H, u, v, H, phi, mask, f_u, f_v, f_H, bed,
                                                           B, beta, gamma, use_forcing != 0, use_mask != 0,
                                                           GRG_PHYS_ARGS, ny, nx, stride, halo);
    return int(cudaGetLastError());
}

int grg_vanka_smooth(int gx, int gy, int bx, int by, float* d_u, float* d_v, float* d_H, float* mask,
                     const float* u, const float* v, const float* H, const float* phi, const float* f_u,
                     const float* f_v, const float* f_H, const float* bed, const float* B, const float* beta,
                     const float* gamma, GRG_PHYS_PARAMS, int ny, int nx, int stride, int halo, int newton_steps,
                     float relaxation, float ssa_damping, float mc_damping, void* s) {
    vanka_smooth<<<d2(gx, gy), d2(bx, by), 0, st(s)>>>(d_u, d_v, d_H, mask, u, v, H, phi, f_u, f_v, f_H, bed, B,
                                                       beta, gamma, GRG_PHYS_ARGS, ny, nx, stride, halo,
                                                       newton_steps, relaxation, ssa_damping, mc_damping);
    return int(cudaGetLastError());
}

int grg_compute_vjp(int gx, int gy, int bx, int by, float* vjp_u, float* vjp_v, float* vjp_H, const float* u,
                    const float* v, const float* H, const float* l_u, const float* l_v, const float* l_H,
                    const float* phi, const float* mask, const float* f_u, const float* f_v, const float* f_H,
                    const float* bed, const float* B, const float* beta, const float* gamma, int use_forcing,
                    int use_mask, GRG_PHYS_PARAMS, int ny, int nx, int stride, int halo, void* s) {
    compute_vjp<<<d2(gx, gy), d2(bx, by), 0, st(s)>>>(vjp_u, vjp_v, vjp_H, u, v, H, l_u, l_v, l_H, phi, mask, f_u,
                                                      f_v, f_H, bed, B, beta, gamma, use_forcing != 0,
                                                      use_mask != 0, GRG_PHYS_ARGS, ny, nx, stride, halo);
    return int(cudaGetLastError());
}

int grg_vanka_smooth_adjoint(int gx, int gy, int bx, int by, float* l_u_out, float* l_v_out, float* l_H_out,
                             const float* u, const float* v, const float* H, const float* phi, const float* mask,
                             const float* r_u, const float* r_v, const float* r_H, const float* bed,
                             const float* B, const float* beta, const float* gamma, GRG_PHYS_PARAMS, int ny, int nx,
                             int stride, int halo, float ssa_damping, float mc_damping, void* s) {
    vanka_smooth_adjoint<<<d2(gx, gy), d2(bx, by), 0, st(s)>>>(l_u_out, l_v_out, l_H_out, u, v, H, phi, mask, r_u,
                                                               r_v, r_H, bed, B, beta, gamma, GRG_PHYS_ARGS, ny, nx,
                                                               stride, halo, ssa_damping, mc_damping);
    return int(cudaGetLastError());
}

int grg_compute_gradient(int which, int gx, int gy, int bx, int by, float* grad, const float* u, const float* v,
                         const float* H, const float* l_u, const float* l_v, const float* l_H, const float* phi,
                         const float* mask, const float* bed, const float* B, const float* beta,
                         const float* gamma, GRG_PHYS_PARAMS, int ny, int nx, int stride, int halo, void* s) {
    if (which == 0)
        compute_gradient_beta<<<d2(gx, gy), d2(bx, by), 0, st(s)>>>(grad, u, v, H, l_u, l_v, l_H, phi, mask, bed,
                                                                    B, beta, gamma, GRG_PHYS_ARGS, ny, nx, stride,
                                                                    halo);
    else
        compute_gradient_bed<<<d2(gx, gy), d2(bx, by), 0, st(s)>>>(grad, u, v, H, l_u, l_v, l_H, phi, mask, bed,
                                                                   B, beta, gamma, GRG_PHYS_ARGS, ny, nx, stride,
                                                                   halo);
    return int(cudaGetLastError());
}

// One transfer kernel of glide/cuda/transfer.cu by name, one-dimensional
// launch of `blocks` x 256 threads as glide/multigrid.py:118-259 does.
int grg_transfer(int op, int blocks, const float* src, float* dst, int ny, int nx, void* s) {
    const dim3 g(unsigned(blocks), 1u, 1u), b(256u, 1u, 1u);
    switch (op) {
        case 0: restrict_vfacet<<<g, b, 0, st(s)>>>(src, dst, ny, nx); break;
        case 1: restrict_hfacet<<<g, b, 0, st(s)>>>(src, dst, ny, nx); break;
        case 2: restrict_cell_avg<<<g, b, 0, st(s)>>>(src, dst, ny, nx); break;
        case 3: restrict_cell_max<<<g, b, 0, st(s)>>>(src, dst, ny, nx); break;
        case 4: prolongate_vfacet_injection<<<g, b, 0, st(s)>>>(src, dst, ny, nx); break;
        case 5: prolongate_vfacet_bilinear<<<g, b, 0, st(s)>>>(src, dst, ny, nx); break;
        case 6: prolongate_cell_injection<<<g, b, 0, st(s)>>>(src, dst, ny, nx); break;
        case 7: prolongate_cell_bilinear<<<g, b, 0, st(s)>>>(src, dst, ny, nx); break;
        default: return int(cudaErrorInvalidValue);
    }
    return int(cudaGetLastError());
}

}  // extern "C"
