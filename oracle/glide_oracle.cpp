// glide_oracle.cpp -- loops of the CPU oracle (TEST INFRASTRUCTURE).
//
// Restates, in this project's own structure, the kernels of the reference
// (JacobDowns/glide):
//   residual          glide/cuda/residuals.cu:6-333
//   vanka sweep       glide/cuda/vanka.cu:91-475 (local system), :478-660 (loop)
//   grounded fraction glide/cuda/viscosity.cu:17-36
//   transpose (VJP)   glide/cuda/residuals.cu:667-1163
//   adjoint vanka     glide/cuda/vanka.cu:663-797
//   gradients         glide/cuda/grad.cu:2-169
//   transfers         glide/cuda/transfer.cu:1-395
// Exported with C linkage as go_<name>_f64 / go_<name>_f32.
#include "glide_oracle.hpp"

#include <vector>

namespace oracle {

// ------------------------------------------------------------------ residual
template <class R>
struct EtaField {
    // Cell viscosity on an extended index range [-2, ny+2) x [-2, nx+2), so
    // that every stencil can look one or two cells past the domain edge.
    int ny, nx;
    std::vector<R> e;
    R at(int i, int j) const { return e[size_t(i + 2) * (nx + 4) + (j + 2)]; }
    void fill(const Level<R>& L, const R* u, const R* v, const Phys<R>& p) {
        ny = L.ny; nx = L.nx;
        e.assign(size_t(ny + 4) * (nx + 4), R(0));
#pragma omp parallel for
        for (int i = -2; i < ny + 2; ++i)
            for (int j = -2; j < nx + 2; ++j)
                e[size_t(i + 2) * (nx + 4) + (j + 2)] = eta_cell(L, u, v, p.n, p.eps_reg, p.dx, i, j);
    }
};

// Mass-balance residual of cell (i, j).  Restates residuals.cu:55-104.
template <class R>
R cell_residual(const Level<R>& L, const Phys<R>& p, bool use_forcing, bool use_mask, int i, int j) {
    const int ny = L.ny, nx = L.nx;
    R dxi = R(1) / p.dx;
    R Hc = L.C(L.H, i, j), phic = L.C(L.phi, i, j);
    R r = Hc / p.dt;
    if (use_forcing) r -= L.C(L.f_H, i, j);
    R Hl = L.C(L.H, i, j - 1), Hr = L.C(L.H, i, j + 1), Ht = L.C(L.H, i - 1, j), Hb = L.C(L.H, i + 1, j);
    R pl = L.C(L.phi, i, j - 1), pr = L.C(L.phi, i, j + 1), pt = L.C(L.phi, i - 1, j), pb = L.C(L.phi, i + 1, j);
    r -= lf_flux(L.U(L.u, i, j), Hl, Hc, j, nx).q * dxi;
    r += facet_calving(Hc, phic, pl, p.calving_rate, (R*)nullptr) * dxi;
    r += lf_flux(L.U(L.u, i, j + 1), Hc, Hr, j + 1, nx).q * dxi;
    r += facet_calving(Hc, phic, pr, p.calving_rate, (R*)nullptr) * dxi;
    r += lf_flux(L.V(L.v, i, j), Hc, Ht, i, ny).q * dxi;
    r += facet_calving(Hc, phic, pt, p.calving_rate, (R*)nullptr) * dxi;
    r -= lf_flux(L.V(L.v, i + 1, j), Hb, Hc, i + 1, ny).q * dxi;
    r += facet_calving(Hc, phic, pb, p.calving_rate, (R*)nullptr) * dxi;
    R msk = use_mask ? L.C(L.mask, i, j) : R(0);
    return (R(1) - msk) * r + msk * (Hc - L.C(L.gamma, i, j));
}

// x-momentum residual on u face (i, j).  Restates residuals.cu:109-219.
template <class R>
R u_residual(const Level<R>& L, const Phys<R>& p, const EtaField<R>& eta, bool use_forcing, int i, int j) {
    const int ny = L.ny, nx = L.nx;
    const R* u = L.u; const R* v = L.v; const R* H = L.H;
    R dxi = R(1) / p.dx;
    R r = 0;
    if (use_forcing) r -= L.U(L.f_u, i, j);
    R Hc = L.C(H, i, j), Hl = L.C(H, i, j - 1);
    R ul = L.U(u, i, j);
    r += sigma_xx(ul, L.U(u, i, j + 1), L.V(v, i, j), L.V(v, i + 1, j), eta.at(i, j) * Hc, dxi, j, nx).s * dxi;
    r -= sigma_xx(L.U(u, i, j - 1), ul, L.V(v, i, j - 1), L.V(v, i + 1, j - 1), eta.at(i, j - 1) * Hl, dxi, j - 1, nx).s * dxi;
    {
        R eH = etaH_vertex(eta.at(i - 1, j - 1), eta.at(i - 1, j), eta.at(i, j - 1), eta.at(i, j),
                           L.C(H, i - 1, j - 1), L.C(H, i - 1, j), Hl, Hc);
        r += sigma_xy(L.U(u, i - 1, j), ul, L.V(v, i, j - 1), L.V(v, i, j), eH, dxi, i, j, ny, nx).s * dxi;
    }
    {
        R eH = etaH_vertex(eta.at(i, j - 1), eta.at(i, j), eta.at(i + 1, j - 1), eta.at(i + 1, j),
                           Hl, Hc, L.C(H, i + 1, j - 1), L.C(H, i + 1, j));
        r -= sigma_xy(ul, L.U(u, i + 1, j), L.V(v, i + 1, j - 1), L.V(v, i + 1, j), eH, dxi, i + 1, j, ny, nx).s * dxi;
    }
    r += tau_basal(ul, L.V(v, i, j - 1), L.V(v, i, j), L.V(v, i + 1, j - 1), L.V(v, i + 1, j),
                   L.C(L.phi, i, j - 1), L.C(L.phi, i, j), L.C(L.beta, i, j - 1), L.C(L.beta, i, j),
                   p.m, p.u_reg, p.water_drag).s;
    r -= tau_driving(Hl, Hc, L.C(L.bed, i, j - 1), L.C(L.bed, i, j), L.C(L.phi, i, j - 1),
                     L.C(L.phi, i, j), dxi, j, nx).s;
    if (j == 0 || j == nx) r = ul;
    return r;
}

// y-momentum residual on v face (i, j).  Restates residuals.cu:221-331.
template <class R>
R v_residual(const Level<R>& L, const Phys<R>& p, const EtaField<R>& eta, bool use_forcing, int i, int j) {
    const int ny = L.ny, nx = L.nx;
    const R* u = L.u; const R* v = L.v; const R* H = L.H;
    R dxi = R(1) / p.dx;
    R r = 0;
    if (use_forcing) r -= L.V(L.f_v, i, j);
    R Hc = L.C(H, i, j), Ht = L.C(H, i - 1, j);
    R vt = L.V(v, i, j);
    r += sigma_yy(L.U(u, i - 1, j), L.U(u, i - 1, j + 1), L.V(v, i - 1, j), vt, eta.at(i - 1, j) * Ht, dxi, i - 1, ny).s * dxi;
    r -= sigma_yy(L.U(u, i, j), L.U(u, i, j + 1), vt, L.V(v, i + 1, j), eta.at(i, j) * Hc, dxi, i, ny).s * dxi;
    {
        R eH = etaH_vertex(eta.at(i - 1, j - 1), eta.at(i - 1, j), eta.at(i, j - 1), eta.at(i, j),
                           L.C(H, i - 1, j - 1), Ht, L.C(H, i, j - 1), Hc);
        r -= sigma_xy(L.U(u, i - 1, j), L.U(u, i, j), L.V(v, i, j - 1), vt, eH, dxi, i, j, ny, nx).s * dxi;
    }
    {
        R eH = etaH_vertex(eta.at(i - 1, j), eta.at(i - 1, j + 1), eta.at(i, j), eta.at(i, j + 1),
                           Ht, L.C(H, i - 1, j + 1), Hc, L.C(H, i, j + 1));
        r += sigma_xy(L.U(u, i - 1, j + 1), L.U(u, i, j + 1), vt, L.V(v, i, j + 1), eH, dxi, i, j + 1, ny, nx).s * dxi;
    }
    r += tau_basal(vt, L.U(u, i - 1, j), L.U(u, i - 1, j + 1), L.U(u, i, j), L.U(u, i, j + 1),
                   L.C(L.phi, i - 1, j), L.C(L.phi, i, j), L.C(L.beta, i - 1, j), L.C(L.beta, i, j),
                   p.m, p.u_reg, p.water_drag).s;
    r -= tau_driving(Hc, Ht, L.C(L.bed, i, j), L.C(L.bed, i - 1, j), L.C(L.phi, i, j),
                     L.C(L.phi, i - 1, j), dxi, i, ny).s;
    if (i == 0 || i == ny) r = vt;
    return r;
}

template <class R>
void residual(const Level<R>& L, const Phys<R>& p, bool use_forcing, bool use_mask, R* r_u, R* r_v, R* r_H) {
    const int ny = L.ny, nx = L.nx;
    EtaField<R> eta;
    eta.fill(L, L.u, L.v, p);
#pragma omp parallel for
    for (int i = 0; i <= ny; ++i) {
        for (int j = 0; j <= nx; ++j) {
            if (i < ny && j < nx) r_H[i * nx + j] = cell_residual(L, p, use_forcing, use_mask, i, j);
            if (i < ny) r_u[i * (nx + 1) + j] = u_residual(L, p, eta, use_forcing, i, j);
            if (j < nx) r_v[i * nx + j] = v_residual(L, p, eta, use_forcing, i, j);
        }
    }
}

// -------------------------------------------------------- local 5x5 system
// Unknowns of cell (i, j): x = (u_l, u_r, v_t, v_b, H_c).  Assembles the
// local Newton matrix J (row-major 5x5) and residual r with every neighbour
// value frozen at the global state and eta frozen.  Restates vanka.cu:91-475.
template <class R>
void local_system(const Level<R>& L, const Phys<R>& p, const EtaField<R>& eta, int i, int j,
                  const R x[5], R J[25], R r[5]) {
    const int ny = L.ny, nx = L.nx;
    const R* u = L.u; const R* v = L.v; const R* H = L.H;
    const R dxi = R(1) / p.dx;
    const R ul = x[0], ur = x[1], vt = x[2], vb = x[3], Hc = x[4];
    for (int k = 0; k < 25; ++k) J[k] = 0;
    for (int k = 0; k < 5; ++k) r[k] = 0;
    const R phc = L.C(L.phi, i, j), phl = L.C(L.phi, i, j - 1), phr = L.C(L.phi, i, j + 1);
    const R pht = L.C(L.phi, i - 1, j), phb = L.C(L.phi, i + 1, j);
    const R Hl = L.C(H, i, j - 1), Hr = L.C(H, i, j + 1), Ht = L.C(H, i - 1, j), Hb = L.C(H, i + 1, j);

    // mass row (vanka.cu:128-194)
    {
        R dc;
        J[24] = R(1) / p.dt;
        r[4] += Hc / p.dt;
        Flux<R> f = lf_flux(ul, Hl, Hc, j, nx);
        J[20] -= f.d_w * dxi; J[24] -= f.d_H1 * dxi; r[4] -= f.q * dxi;
        R c = facet_calving(Hc, phc, phl, p.calving_rate, &dc);
        J[24] += dc * dxi; r[4] += c * dxi;
        f = lf_flux(ur, Hc, Hr, j + 1, nx);
        J[21] += f.d_w * dxi; J[24] += f.d_H0 * dxi; r[4] += f.q * dxi;
        c = facet_calving(Hc, phc, phr, p.calving_rate, &dc);
        J[24] += dc * dxi; r[4] += c * dxi;
        f = lf_flux(vt, Hc, Ht, i, ny);
        J[22] += f.d_w * dxi; J[24] += f.d_H0 * dxi; r[4] += f.q * dxi;
        c = facet_calving(Hc, phc, pht, p.calving_rate, &dc);
        J[24] += dc * dxi; r[4] += c * dxi;
        f = lf_flux(vb, Hb, Hc, i + 1, ny);
        J[23] -= f.d_w * dxi; J[24] -= f.d_H1 * dxi; r[4] -= f.q * dxi;
        c = facet_calving(Hc, phc, phb, p.calving_rate, &dc);
        J[24] += dc * dxi; r[4] += c * dxi;
    }
    const R ec = eta.at(i, j);
    // normal stresses of the cell itself act on all four faces (vanka.cu:196-239)
    {
        Normal<R> s = sigma_xx(ul, ur, vt, vb, ec * Hc, dxi, j, nx);
        r[0] += s.s * dxi;
        J[0] += s.d_ul * dxi; J[1] += s.d_ur * dxi; J[2] += s.d_vt * dxi; J[3] += s.d_vb * dxi;
        J[4] += s.d_etaH * ec * dxi;
        r[1] -= s.s * dxi;
        J[5] -= s.d_ul * dxi; J[6] -= s.d_ur * dxi; J[7] -= s.d_vt * dxi; J[8] -= s.d_vb * dxi;
        J[9] -= s.d_etaH * ec * dxi;
        Normal<R> t = sigma_yy(ul, ur, vt, vb, ec * Hc, dxi, i, ny);
        r[2] -= t.s * dxi;
        J[10] -= t.d_ul * dxi; J[11] -= t.d_ur * dxi; J[12] -= t.d_vt * dxi; J[13] -= t.d_vb * dxi;
        J[14] -= t.d_etaH * ec * dxi;
        r[3] += t.s * dxi;
        J[15] += t.d_ul * dxi; J[16] += t.d_ur * dxi; J[17] += t.d_vt * dxi; J[18] += t.d_vb * dxi;
        J[19] += t.d_etaH * ec * dxi;
    }
    // normal stresses of the four neighbours on the shared face (vanka.cu:241-296)
    {
        Normal<R> s = sigma_xx(L.U(u, i, j - 1), ul, L.V(v, i, j - 1), L.V(v, i + 1, j - 1),
                               eta.at(i, j - 1) * Hl, dxi, j - 1, nx);
        r[0] -= s.s * dxi; J[0] -= s.d_ur * dxi;
        s = sigma_xx(ur, L.U(u, i, j + 2), L.V(v, i, j + 1), L.V(v, i + 1, j + 1),
                     eta.at(i, j + 1) * Hr, dxi, j + 1, nx);
        r[1] += s.s * dxi; J[6] += s.d_ul * dxi;
        s = sigma_yy(L.U(u, i - 1, j), L.U(u, i - 1, j + 1), L.V(v, i - 1, j), vt,
                     eta.at(i - 1, j) * Ht, dxi, i - 1, ny);
        r[2] += s.s * dxi; J[12] += s.d_vb * dxi;
        s = sigma_yy(L.U(u, i + 1, j), L.U(u, i + 1, j + 1), vb, L.V(v, i + 2, j),
                     eta.at(i + 1, j) * Hb, dxi, i + 1, ny);
        r[3] -= s.s * dxi; J[18] -= s.d_vt * dxi;
    }
    // shear stress on the four corners (vanka.cu:299-400)
    {
        R q = R(0.25) * ec;  // d(vertex eta*H)/dH_c
        R eH = etaH_vertex(eta.at(i - 1, j - 1), eta.at(i - 1, j), eta.at(i, j - 1), ec,
                           L.C(H, i - 1, j - 1), Ht, Hl, Hc);
        Shear<R> s = sigma_xy(L.U(u, i - 1, j), ul, L.V(v, i, j - 1), vt, eH, dxi, i, j, ny, nx);
        r[0] += s.s * dxi; J[0] += s.d_ub * dxi; J[4] += s.d_etaH * q * dxi;
        r[2] -= s.s * dxi; J[12] -= s.d_vr * dxi; J[14] -= s.d_etaH * q * dxi;

        eH = etaH_vertex(eta.at(i - 1, j), eta.at(i - 1, j + 1), ec, eta.at(i, j + 1),
                         Ht, L.C(H, i - 1, j + 1), Hc, Hr);
        s = sigma_xy(L.U(u, i - 1, j + 1), ur, vt, L.V(v, i, j + 1), eH, dxi, i, j + 1, ny, nx);
        r[1] += s.s * dxi; J[6] += s.d_ub * dxi; J[9] += s.d_etaH * q * dxi;
        r[2] += s.s * dxi; J[12] += s.d_vl * dxi; J[14] += s.d_etaH * q * dxi;

        eH = etaH_vertex(eta.at(i, j - 1), ec, eta.at(i + 1, j - 1), eta.at(i + 1, j),
                         Hl, Hc, L.C(H, i + 1, j - 1), Hb);
        s = sigma_xy(ul, L.U(u, i + 1, j), L.V(v, i + 1, j - 1), vb, eH, dxi, i + 1, j, ny, nx);
        r[0] -= s.s * dxi; J[0] -= s.d_ut * dxi; J[4] -= s.d_etaH * q * dxi;
        r[3] -= s.s * dxi; J[18] -= s.d_vr * dxi; J[19] -= s.d_etaH * q * dxi;

        eH = etaH_vertex(ec, eta.at(i, j + 1), eta.at(i + 1, j), eta.at(i + 1, j + 1),
                         Hc, Hr, Hb, L.C(H, i + 1, j + 1));
        s = sigma_xy(ur, L.U(u, i + 1, j + 1), vb, L.V(v, i + 1, j + 1), eH, dxi, i + 1, j + 1, ny, nx);
        r[1] -= s.s * dxi; J[6] -= s.d_ut * dxi; J[9] -= s.d_etaH * q * dxi;
        r[3] += s.s * dxi; J[18] += s.d_vl * dxi; J[19] += s.d_etaH * q * dxi;
    }
    // basal drag on the four faces (vanka.cu:403-461); H-derivatives are zero
    {
        const R bc = L.C(L.beta, i, j);
        Basal<R> b = tau_basal(ul, L.V(v, i, j - 1), vt, L.V(v, i + 1, j - 1), vb, phl, phc,
                               L.C(L.beta, i, j - 1), bc, p.m, p.u_reg, p.water_drag);
        r[0] += b.s; J[0] += b.d_w; J[2] += b.d_b; J[3] += b.d_d;
        b = tau_basal(ur, vt, L.V(v, i, j + 1), vb, L.V(v, i + 1, j + 1), phc, phr, bc,
                      L.C(L.beta, i, j + 1), p.m, p.u_reg, p.water_drag);
        r[1] += b.s; J[6] += b.d_w; J[7] += b.d_a; J[8] += b.d_c;
        b = tau_basal(vt, L.U(u, i - 1, j), L.U(u, i - 1, j + 1), ul, ur, pht, phc,
                      L.C(L.beta, i - 1, j), bc, p.m, p.u_reg, p.water_drag);
        r[2] += b.s; J[12] += b.d_w; J[10] += b.d_c; J[11] += b.d_d;
        b = tau_basal(vb, ul, ur, L.U(u, i + 1, j), L.U(u, i + 1, j + 1), phc, phb, bc,
                      L.C(L.beta, i + 1, j), p.m, p.u_reg, p.water_drag);
        r[3] += b.s; J[18] += b.d_w; J[15] += b.d_a; J[16] += b.d_b;
    }
    // driving stress on the four faces (vanka.cu:464-474 and :405-445 of stress.cu)
    {
        const R bdc = L.C(L.bed, i, j);
        Driving<R> d = tau_driving(Hl, Hc, L.C(L.bed, i, j - 1), bdc, phl, phc, dxi, j, nx);
        r[0] -= d.s; J[4] -= d.d_H1;
        d = tau_driving(Hc, Hr, bdc, L.C(L.bed, i, j + 1), phc, phr, dxi, j + 1, nx);
        r[1] -= d.s; J[9] -= d.d_H0;
        d = tau_driving(Hc, Ht, bdc, L.C(L.bed, i - 1, j), phc, pht, dxi, i, ny);
        r[2] -= d.s; J[14] -= d.d_H0;
        d = tau_driving(Hb, Hc, L.C(L.bed, i + 1, j), bdc, phb, phc, dxi, i + 1, ny);
        r[3] -= d.s; J[19] -= d.d_H1;
    }
}

// Doolittle LU without pivoting followed by the two triangular solves, in the
// operation order of vanka.cu:5-48.
template <class R>
void lu5_solve(const R A[25], const R b[5], R x[5]) {
    R LU[5][5];
    for (int a = 0; a < 5; ++a)
        for (int c = 0; c < 5; ++c) LU[a][c] = A[a * 5 + c];
    for (int k = 0; k < 5; ++k) {
        R inv = R(1) / LU[k][k];
        for (int a = k + 1; a < 5; ++a) {
            LU[a][k] *= inv;
            for (int c = k + 1; c < 5; ++c) LU[a][c] -= LU[a][k] * LU[k][c];
        }
    }
    R y[5];
    y[0] = b[0];
    y[1] = b[1] - LU[1][0] * y[0];
    y[2] = b[2] - LU[2][0] * y[0] - LU[2][1] * y[1];
    y[3] = b[3] - LU[3][0] * y[0] - LU[3][1] * y[1] - LU[3][2] * y[2];
    y[4] = b[4] - LU[4][0] * y[0] - LU[4][1] * y[1] - LU[4][2] * y[2] - LU[4][3] * y[3];
    x[4] = y[4] / LU[4][4];
    x[3] = (y[3] - LU[3][4] * x[4]) / LU[3][3];
    x[2] = (y[2] - LU[2][3] * x[3] - LU[2][4] * x[4]) / LU[2][2];
    x[1] = (y[1] - LU[1][2] * x[2] - LU[1][3] * x[3] - LU[1][4] * x[4]) / LU[1][1];
    x[0] = (y[0] - LU[0][1] * x[1] - LU[0][2] * x[2] - LU[0][3] * x[3] - LU[0][4] * x[4]) / LU[0][0];
}

// Replace row and column k of the local system by the identity row.
template <class R>
inline void pin_row(R J[25], int k) {
    for (int c = 0; c < 5; ++c) J[k * 5 + c] = 0;
    for (int a = 0; a < 5; ++a) J[a * 5 + k] = 0;
    J[k * 5 + k] = 1;
}

struct NewtonCfg { int steps; double ssa_damping, mc_damping; };

// One additive Vanka pass: every cell runs its damped local Newton iteration
// against the frozen global state; the face corrections of the two cells
// sharing a face are averaged.  Outputs delta_u, delta_v, delta_H and the new
// active-set mask, exactly what the reference's kernel leaves in its delta
// buffers.  Restates vanka.cu:478-660; `newton_iters`, if given, receives the
// iteration count of each cell.
template <class R>
void vanka(const Level<R>& L, const Phys<R>& p, NewtonCfg cfg, R* d_u, R* d_v, R* d_H, R* mask_out,
           int* newton_iters) {
    const int ny = L.ny, nx = L.nx;
    EtaField<R> eta;
    eta.fill(L, L.u, L.v, p);
    std::vector<R> cell_d(size_t(ny) * nx * 4);
    const R tol = R(kNewtonTol);
#pragma omp parallel for
    for (int i = 0; i < ny; ++i) {
        for (int j = 0; j < nx; ++j) {
            R x[5] = {L.U(L.u, i, j), L.U(L.u, i, j + 1), L.V(L.v, i, j), L.V(L.v, i + 1, j), L.C(L.H, i, j)};
            const R x0[5] = {x[0], x[1], x[2], x[3], x[4]};
            const R thk = L.C(L.gamma, i, j);
            R masked = L.C(L.mask, i, j);
            R comp[5] = {0, 0, 0, 0, 0};
            R rnorm = 1;
            int k = 0;
            R J[25], r[5];
            while (k < cfg.steps && rnorm > tol) {
                local_system(L, p, eta, i, j, x, J, r);
                r[0] -= L.U(L.f_u, i, j);
                r[1] -= L.U(L.f_u, i, j + 1);
                r[2] -= L.V(L.f_v, i, j);
                r[3] -= L.V(L.f_v, i + 1, j);
                r[4] -= L.C(L.f_H, i, j);
                J[0] -= R(cfg.ssa_damping); J[6] -= R(cfg.ssa_damping);
                J[12] -= R(cfg.ssa_damping); J[18] -= R(cfg.ssa_damping);
                J[24] += R(cfg.mc_damping);
                if (j == 0) { pin_row(J, 0); r[0] = x[0]; }
                if (j == nx - 1) { pin_row(J, 1); r[1] = x[1]; }
                if (i == 0) { pin_row(J, 2); r[2] = x[2]; }
                if (i == ny - 1) { pin_row(J, 3); r[3] = x[3]; }
                if ((x[4] - p.dt * r[4]) <= thk) {
                    masked = 1;
                    pin_row(J, 4);
                    r[4] = x[4] - thk;
                } else {
                    masked = 0;
                }
                R dx[5];
                lu5_solve(J, r, dx);
                rnorm = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3] + r[4] * r[4];
                const R relax = R(0.5);  // fixed inside the reference kernel (vanka.cu:615)
                for (int q = 0; q < 5; ++q) {  // compensated update, vanka.cu:617-640
                    R y = -relax * dx[q] - comp[q];
                    R t = x[q] + y;
                    comp[q] = (t - x[q]) - y;
                    x[q] = t;
                }
                x[4] = std::max(x[4], thk);
                ++k;
            }
            R* cd = &cell_d[(size_t(i) * nx + j) * 4];
            for (int q = 0; q < 4; ++q) cd[q] = R(0.5) * (x[q] - x0[q]);
            d_H[i * nx + j] = x[4] - x0[4];
            mask_out[i * nx + j] = masked;
            if (newton_iters) newton_iters[i * nx + j] = k;
        }
    }
    // every face sums the half-corrections of the cells on either side
#pragma omp parallel for
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j <= nx; ++j) {
            R s = 0;
            if (j > 0) s += cell_d[(size_t(i) * nx + j - 1) * 4 + 1];
            if (j < nx) s += cell_d[(size_t(i) * nx + j) * 4 + 0];
            d_u[i * (nx + 1) + j] = s;
        }
#pragma omp parallel for
    for (int i = 0; i <= ny; ++i)
        for (int j = 0; j < nx; ++j) {
            R s = 0;
            if (i > 0) s += cell_d[(size_t(i - 1) * nx + j) * 4 + 3];
            if (i < ny) s += cell_d[(size_t(i) * nx + j) * 4 + 2];
            d_v[i * nx + j] = s;
        }
}

// Per-cell Newton matrix and residual after damping, boundary rows and the
// active set, as the reference's debug kernel writes them.  Restates
// vanka.cu:801-908 (no damping there).
template <class R>
void vanka_dump(const Level<R>& L, const Phys<R>& p, R* Jout, R* rout) {
    const int ny = L.ny, nx = L.nx;
    EtaField<R> eta;
    eta.fill(L, L.u, L.v, p);
#pragma omp parallel for
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) {
            R x[5] = {L.U(L.u, i, j), L.U(L.u, i, j + 1), L.V(L.v, i, j), L.V(L.v, i + 1, j), L.C(L.H, i, j)};
            const R thk = L.C(L.gamma, i, j);
            R J[25], r[5];
            local_system(L, p, eta, i, j, x, J, r);
            r[0] -= L.U(L.f_u, i, j); r[1] -= L.U(L.f_u, i, j + 1);
            r[2] -= L.V(L.f_v, i, j); r[3] -= L.V(L.f_v, i + 1, j);
            r[4] -= L.C(L.f_H, i, j);
            if (j == 0) { pin_row(J, 0); r[0] = x[0]; }
            if (j == nx - 1) { pin_row(J, 1); r[1] = x[1]; }
            if (i == 0) { pin_row(J, 2); r[2] = x[2]; }
            if (i == ny - 1) { pin_row(J, 3); r[3] = x[3]; }
            if ((x[4] - p.dt * r[4]) <= thk) { pin_row(J, 4); r[4] = x[4] - thk; }
            for (int k = 0; k < 25; ++k) Jout[(size_t(i) * nx + j) * 25 + k] = J[k];
            for (int k = 0; k < 5; ++k) rout[(size_t(i) * nx + j) * 5 + k] = r[k];
        }
}

// -------------------------------------------------------------- grounding
template <class R>
void compute_grounded(int ny, int nx, R* phi, const R* H, const R* bed, R c, R relax) {
#pragma omp parallel for
    for (int k = 0; k < ny * nx; ++k)
        phi[k] = (R(1) - relax) * grounded(H[k], bed[k], c) + relax * phi[k];
}

// ------------------------------------------------------------ transpose (VJP)
// lambda^T dR/dx (minus the forcing when use_forcing), scattered from every
// residual row onto the unknowns it depends on, then filtered per target:
// u faces on x = 0 / x = nx and v faces on y = 0 / y = ny receive nothing,
// and cells with mask > 0 receive nothing.  The momentum rows apply the
// forward derivative of eta along lambda (the viscous block is symmetric).
// Restates residuals.cu:667-1163.
template <class R>
void vjp(const Level<R>& L, const Phys<R>& p, const R* lu, const R* lv, const R* lH, bool use_forcing,
         R* out_u, R* out_v, R* out_H) {
    const int ny = L.ny, nx = L.nx;
    const R* u = L.u; const R* v = L.v; const R* H = L.H;
    const R dxi = R(1) / p.dx;
    // viscosity and its derivative along lambda on [-2, ny+2) x [-2, nx+2)
    const int W = nx + 4;
    std::vector<R> ev(size_t(ny + 4) * W), ed(size_t(ny + 4) * W);
#pragma omp parallel for
    for (int i = -2; i < ny + 2; ++i)
        for (int j = -2; j < nx + 2; ++j) {
            ev[size_t(i + 2) * W + j + 2] = eta_cell(L, u, v, p.n, p.eps_reg, p.dx, i, j);
            ed[size_t(i + 2) * W + j + 2] = eta_cell_dot(L, u, v, lu, lv, p.n, p.eps_reg, p.dx, i, j);
        }
    auto E = [&](int i, int j) { return ev[size_t(i + 2) * W + j + 2]; };
    auto D = [&](int i, int j) { return ed[size_t(i + 2) * W + j + 2]; };
    // accumulators over [-1, ny+1] x [-1, nx+2] so out-of-domain targets have a slot
    const int AW = nx + 4;
    std::vector<R> au(size_t(ny + 3) * AW, 0), av(size_t(ny + 3) * AW, 0), aH(size_t(ny + 3) * AW, 0);
    auto AU = [&](int i, int j) -> R& { return au[size_t(i + 1) * AW + j + 1]; };
    auto AV = [&](int i, int j) -> R& { return av[size_t(i + 1) * AW + j + 1]; };
    auto AH = [&](int i, int j) -> R& { return aH[size_t(i + 1) * AW + j + 1]; };
    auto Hs = [&](int i, int j) { return L.C(H, i, j); };

    for (int i = 0; i <= ny; ++i) {
        for (int j = 0; j <= nx; ++j) {
            const bool has_cell = i < ny && j < nx;
            const bool has_u = i < ny;
            const bool has_v = j < nx;
            if (has_cell) {
                R Hc = Hs(i, j), Hl = Hs(i, j - 1), Hr = Hs(i, j + 1), Ht = Hs(i - 1, j), Hb = Hs(i + 1, j);
                R phc = L.C(L.phi, i, j);
                R lam = L.C(lH, i, j) * (R(1) - L.C(L.mask, i, j));
                R dc;
                AH(i, j) += lam / p.dt;
                Flux<R> f = lf_flux(L.U(u, i, j), Hl, Hc, j, nx);
                AH(i, j) += -lam * f.d_H1 * dxi; AH(i, j - 1) += -lam * f.d_H0 * dxi; AU(i, j) += -lam * f.d_w * dxi;
                facet_calving(Hc, phc, L.C(L.phi, i, j - 1), p.calving_rate, &dc);
                AH(i, j) += lam * dc * dxi;
                f = lf_flux(L.U(u, i, j + 1), Hc, Hr, j + 1, nx);
                AH(i, j) += lam * f.d_H0 * dxi; AH(i, j + 1) += lam * f.d_H1 * dxi; AU(i, j + 1) += lam * f.d_w * dxi;
                facet_calving(Hc, phc, L.C(L.phi, i, j + 1), p.calving_rate, &dc);
                AH(i, j) += lam * dc * dxi;
                f = lf_flux(L.V(v, i, j), Hc, Ht, i, ny);
                AH(i, j) += lam * f.d_H0 * dxi; AH(i - 1, j) += lam * f.d_H1 * dxi; AV(i, j) += lam * f.d_w * dxi;
                facet_calving(Hc, phc, L.C(L.phi, i - 1, j), p.calving_rate, &dc);
                AH(i, j) += lam * dc * dxi;
                f = lf_flux(L.V(v, i + 1, j), Hb, Hc, i + 1, ny);
                AH(i, j) += -lam * f.d_H1 * dxi; AH(i + 1, j) += -lam * f.d_H0 * dxi; AV(i + 1, j) += -lam * f.d_w * dxi;
                facet_calving(Hc, phc, L.C(L.phi, i + 1, j), p.calving_rate, &dc);
                AH(i, j) += lam * dc * dxi;
                if (use_forcing) AH(i, j) += -L.C(L.f_H, i, j);
            }
            if (has_u) {
                R Hc = Hs(i, j), Hl = Hs(i, j - 1);
                R ul = L.U(u, i, j);
                R lul = L.U(lu, i, j);
                {   // sigma_xx of cell (i, j)
                    R ur = L.U(u, i, j + 1), vt = L.V(v, i, j), vb = L.V(v, i + 1, j);
                    Normal<R> s = sigma_xx(ul, ur, vt, vb, E(i, j) * Hc, dxi, j, nx);
                    R a = s.d_ul * lul + s.d_ur * L.U(lu, i, j + 1) + s.d_vt * L.V(lv, i, j) +
                          s.d_vb * L.V(lv, i + 1, j) + s.d_etaH * (Hc * D(i, j));
                    AU(i, j) += a * dxi;
                    AH(i, j) += lul * s.d_etaH * E(i, j) * dxi;
                }
                {   // sigma_xx of cell (i, j-1)
                    Normal<R> s = sigma_xx(L.U(u, i, j - 1), ul, L.V(v, i, j - 1), L.V(v, i + 1, j - 1),
                                           E(i, j - 1) * Hl, dxi, j - 1, nx);
                    R a = s.d_ul * L.U(lu, i, j - 1) + s.d_ur * lul + s.d_vt * L.V(lv, i, j - 1) +
                          s.d_vb * L.V(lv, i + 1, j - 1) + s.d_etaH * (Hl * D(i, j - 1));
                    AU(i, j) += -a * dxi;
                    AH(i, j - 1) += -lul * s.d_etaH * E(i, j - 1) * dxi;
                }
                {   // sigma_xy at vertex (i, j)
                    R Htl = Hs(i - 1, j - 1), Ht = Hs(i - 1, j);
                    R eH = etaH_vertex(E(i - 1, j - 1), E(i - 1, j), E(i, j - 1), E(i, j), Htl, Ht, Hl, Hc);
                    R deH = R(0.25) * Htl * D(i - 1, j - 1) + R(0.25) * Ht * D(i - 1, j) +
                            R(0.25) * Hl * D(i, j - 1) + R(0.25) * Hc * D(i, j);
                    Shear<R> s = sigma_xy(L.U(u, i - 1, j), ul, L.V(v, i, j - 1), L.V(v, i, j), eH, dxi, i, j, ny, nx);
                    R a = s.d_ut * L.U(lu, i - 1, j) + s.d_ub * lul + s.d_vl * L.V(lv, i, j - 1) +
                          s.d_vr * L.V(lv, i, j) + s.d_etaH * deH;
                    AU(i, j) += a * dxi;
                    R g = lul * s.d_etaH;
                    AH(i - 1, j - 1) += g * R(0.25) * E(i - 1, j - 1) * dxi;
                    AH(i - 1, j) += g * R(0.25) * E(i - 1, j) * dxi;
                    AH(i, j - 1) += g * R(0.25) * E(i, j - 1) * dxi;
                    AH(i, j) += g * R(0.25) * E(i, j) * dxi;
                }
                {   // sigma_xy at vertex (i+1, j)
                    R Hbl = Hs(i + 1, j - 1), Hb = Hs(i + 1, j);
                    R eH = etaH_vertex(E(i, j - 1), E(i, j), E(i + 1, j - 1), E(i + 1, j), Hl, Hc, Hbl, Hb);
                    R deH = R(0.25) * Hl * D(i, j - 1) + R(0.25) * Hc * D(i, j) +
                            R(0.25) * Hbl * D(i + 1, j - 1) + R(0.25) * Hb * D(i + 1, j);
                    Shear<R> s = sigma_xy(ul, L.U(u, i + 1, j), L.V(v, i + 1, j - 1), L.V(v, i + 1, j), eH, dxi,
                                          i + 1, j, ny, nx);
                    R a = s.d_ut * lul + s.d_ub * L.U(lu, i + 1, j) + s.d_vl * L.V(lv, i + 1, j - 1) +
                          s.d_vr * L.V(lv, i + 1, j) + s.d_etaH * deH;
                    AU(i, j) += -a * dxi;
                    R g = lul * s.d_etaH;
                    AH(i, j - 1) += -g * R(0.25) * E(i, j - 1) * dxi;
                    AH(i, j) += -g * R(0.25) * E(i, j) * dxi;
                    AH(i + 1, j - 1) += -g * R(0.25) * E(i + 1, j - 1) * dxi;
                    AH(i + 1, j) += -g * R(0.25) * E(i + 1, j) * dxi;
                }
                {   // basal drag
                    Basal<R> b = tau_basal(ul, L.V(v, i, j - 1), L.V(v, i, j), L.V(v, i + 1, j - 1), L.V(v, i + 1, j),
                                           L.C(L.phi, i, j - 1), L.C(L.phi, i, j), L.C(L.beta, i, j - 1),
                                           L.C(L.beta, i, j), p.m, p.u_reg, p.water_drag);
                    AU(i, j) += lul * b.d_w;
                    AV(i, j - 1) += lul * b.d_a; AV(i, j) += lul * b.d_b;
                    AV(i + 1, j - 1) += lul * b.d_c; AV(i + 1, j) += lul * b.d_d;
                }
                {   // driving stress
                    Driving<R> d = tau_driving(Hl, Hc, L.C(L.bed, i, j - 1), L.C(L.bed, i, j), L.C(L.phi, i, j - 1),
                                               L.C(L.phi, i, j), dxi, j, nx);
                    AH(i, j - 1) += -lul * d.d_H0;
                    AH(i, j) += -lul * d.d_H1;
                }
                if (use_forcing) AU(i, j) += -L.U(L.f_u, i, j);
            }
            if (has_v) {
                R Hc = Hs(i, j), Ht = Hs(i - 1, j);
                R vt = L.V(v, i, j);
                R lvt = L.V(lv, i, j);
                {   // sigma_yy of cell (i-1, j)
                    Normal<R> s = sigma_yy(L.U(u, i - 1, j), L.U(u, i - 1, j + 1), L.V(v, i - 1, j), vt,
                                           E(i - 1, j) * Ht, dxi, i - 1, ny);
                    R a = s.d_ul * L.U(lu, i - 1, j) + s.d_ur * L.U(lu, i - 1, j + 1) + s.d_vt * L.V(lv, i - 1, j) +
                          s.d_vb * lvt + s.d_etaH * (Ht * D(i - 1, j));
                    AV(i, j) += a * dxi;
                    AH(i - 1, j) += lvt * s.d_etaH * E(i - 1, j) * dxi;
                }
                {   // sigma_yy of cell (i, j)
                    Normal<R> s = sigma_yy(L.U(u, i, j), L.U(u, i, j + 1), vt, L.V(v, i + 1, j), E(i, j) * Hc, dxi, i, ny);
                    R a = s.d_ul * L.U(lu, i, j) + s.d_ur * L.U(lu, i, j + 1) + s.d_vt * lvt +
                          s.d_vb * L.V(lv, i + 1, j) + s.d_etaH * (Hc * D(i, j));
                    AV(i, j) += -a * dxi;
                    AH(i, j) += -lvt * s.d_etaH * E(i, j) * dxi;
                }
                {   // sigma_xy at vertex (i, j)
                    R Htl = Hs(i - 1, j - 1), Hl = Hs(i, j - 1);
                    R eH = etaH_vertex(E(i - 1, j - 1), E(i - 1, j), E(i, j - 1), E(i, j), Htl, Ht, Hl, Hc);
                    R deH = R(0.25) * Htl * D(i - 1, j - 1) + R(0.25) * Ht * D(i - 1, j) +
                            R(0.25) * Hl * D(i, j - 1) + R(0.25) * Hc * D(i, j);
                    Shear<R> s = sigma_xy(L.U(u, i - 1, j), L.U(u, i, j), L.V(v, i, j - 1), vt, eH, dxi, i, j, ny, nx);
                    R a = s.d_ut * L.U(lu, i - 1, j) + s.d_ub * L.U(lu, i, j) + s.d_vl * L.V(lv, i, j - 1) +
                          s.d_vr * lvt + s.d_etaH * deH;
                    AV(i, j) += -a * dxi;
                    R g = lvt * s.d_etaH;
                    AH(i - 1, j - 1) += -g * R(0.25) * E(i - 1, j - 1) * dxi;
                    AH(i - 1, j) += -g * R(0.25) * E(i - 1, j) * dxi;
                    AH(i, j - 1) += -g * R(0.25) * E(i, j - 1) * dxi;
                    AH(i, j) += -g * R(0.25) * E(i, j) * dxi;
                }
                {   // sigma_xy at vertex (i, j+1)
                    R Htr = Hs(i - 1, j + 1), Hr = Hs(i, j + 1);
                    R eH = etaH_vertex(E(i - 1, j), E(i - 1, j + 1), E(i, j), E(i, j + 1), Ht, Htr, Hc, Hr);
                    R deH = R(0.25) * Ht * D(i - 1, j) + R(0.25) * Htr * D(i - 1, j + 1) +
                            R(0.25) * Hc * D(i, j) + R(0.25) * Hr * D(i, j + 1);
                    Shear<R> s = sigma_xy(L.U(u, i - 1, j + 1), L.U(u, i, j + 1), vt, L.V(v, i, j + 1), eH, dxi,
                                          i, j + 1, ny, nx);
                    R a = s.d_ut * L.U(lu, i - 1, j + 1) + s.d_ub * L.U(lu, i, j + 1) + s.d_vl * lvt +
                          s.d_vr * L.V(lv, i, j + 1) + s.d_etaH * deH;
                    AV(i, j) += a * dxi;
                    R g = lvt * s.d_etaH;
                    AH(i - 1, j) += g * R(0.25) * E(i - 1, j) * dxi;
                    AH(i - 1, j + 1) += g * R(0.25) * E(i - 1, j + 1) * dxi;
                    AH(i, j) += g * R(0.25) * E(i, j) * dxi;
                    AH(i, j + 1) += g * R(0.25) * E(i, j + 1) * dxi;
                }
                {   // basal drag
                    Basal<R> b = tau_basal(vt, L.U(u, i - 1, j), L.U(u, i - 1, j + 1), L.U(u, i, j), L.U(u, i, j + 1),
                                           L.C(L.phi, i - 1, j), L.C(L.phi, i, j), L.C(L.beta, i - 1, j),
                                           L.C(L.beta, i, j), p.m, p.u_reg, p.water_drag);
                    AV(i, j) += lvt * b.d_w;
                    AU(i - 1, j) += lvt * b.d_a; AU(i - 1, j + 1) += lvt * b.d_b;
                    AU(i, j) += lvt * b.d_c; AU(i, j + 1) += lvt * b.d_d;
                }
                {   // driving stress
                    Driving<R> d = tau_driving(Hc, Ht, L.C(L.bed, i, j), L.C(L.bed, i - 1, j), L.C(L.phi, i, j),
                                               L.C(L.phi, i - 1, j), dxi, i, ny);
                    AH(i - 1, j) += -lvt * d.d_H1;
                    AH(i, j) += -lvt * d.d_H0;
                }
                if (use_forcing) AV(i, j) += -L.V(L.f_v, i, j);
            }
        }
    }
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j <= nx; ++j) out_u[i * (nx + 1) + j] = (j > 0 && j < nx) ? AU(i, j) : R(0);
    for (int i = 0; i <= ny; ++i)
        for (int j = 0; j < nx; ++j) out_v[i * nx + j] = (i > 0 && i < ny) ? AV(i, j) : R(0);
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) out_H[i * nx + j] = L.C(L.mask, i, j) > R(0) ? R(0) : AH(i, j);
}

// Adjoint block smoother: the same local Newton matrix at the forward state
// (with damping, boundary rows and the stored active set), transposed and
// solved against the adjoint residual; half of each face correction goes to
// each of the two cells sharing the face.  Restates vanka.cu:663-797.
template <class R>
void vanka_adjoint(const Level<R>& L, const Phys<R>& p, double ssa_damping, double mc_damping,
                   const R* ru, const R* rv, const R* rH, R* d_u, R* d_v, R* d_H) {
    const int ny = L.ny, nx = L.nx;
    EtaField<R> eta;
    eta.fill(L, L.u, L.v, p);
    std::vector<R> cell_d(size_t(ny) * nx * 4);
#pragma omp parallel for
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) {
            R x[5] = {L.U(L.u, i, j), L.U(L.u, i, j + 1), L.V(L.v, i, j), L.V(L.v, i + 1, j), L.C(L.H, i, j)};
            R J[25], rr[5];
            local_system(L, p, eta, i, j, x, J, rr);
            J[0] -= R(ssa_damping); J[6] -= R(ssa_damping); J[12] -= R(ssa_damping); J[18] -= R(ssa_damping);
            J[24] += R(mc_damping);
            R b[5] = {L.U(ru, i, j), L.U(ru, i, j + 1), L.V(rv, i, j), L.V(rv, i + 1, j), L.C(rH, i, j)};
            if (j == 0) { pin_row(J, 0); b[0] = 0; }
            if (j == nx - 1) { pin_row(J, 1); b[1] = 0; }
            if (i == 0) { pin_row(J, 2); b[2] = 0; }
            if (i == ny - 1) { pin_row(J, 3); b[3] = 0; }
            if (L.C(L.mask, i, j) > R(0.5)) { pin_row(J, 4); b[4] = 0; }
            R JT[25];
            for (int a = 0; a < 5; ++a)
                for (int c = 0; c < 5; ++c) JT[a * 5 + c] = J[c * 5 + a];
            R dl[5];
            lu5_solve(JT, b, dl);
            R* cd = &cell_d[(size_t(i) * nx + j) * 4];
            for (int q = 0; q < 4; ++q) cd[q] = R(0.5) * dl[q];
            d_H[i * nx + j] = dl[4];
        }
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j <= nx; ++j) {
            R s = 0;
            if (j > 0) s += cell_d[(size_t(i) * nx + j - 1) * 4 + 1];
            if (j < nx) s += cell_d[(size_t(i) * nx + j) * 4 + 0];
            d_u[i * (nx + 1) + j] = s;
        }
    for (int i = 0; i <= ny; ++i)
        for (int j = 0; j < nx; ++j) {
            R s = 0;
            if (i > 0) s += cell_d[(size_t(i - 1) * nx + j) * 4 + 3];
            if (i < ny) s += cell_d[(size_t(i) * nx + j) * 4 + 2];
            d_v[i * nx + j] = s;
        }
}

// d(lambda^T R)/d(beta) and d(lambda^T R)/d(bed) through basal and driving
// stress; the reference's index guards (j > 0, j < nx-1, i > 0, i < ny-1)
// are kept.  Restates grad.cu:2-88 and :91-169.
template <class R>
void gradients(const Level<R>& L, const Phys<R>& p, const R* lu, const R* lv, R* g_beta, R* g_bed) {
    const int ny = L.ny, nx = L.nx;
    const R* u = L.u; const R* v = L.v; const R* H = L.H;
    const R dxi = R(1) / p.dx;
    if (g_beta) std::fill(g_beta, g_beta + size_t(ny) * nx, R(0));
    if (g_bed) std::fill(g_bed, g_bed + size_t(ny) * nx, R(0));
    for (int i = 0; i <= ny; ++i)
        for (int j = 0; j <= nx; ++j) {
            if (i < ny) {
                R lul = L.U(lu, i, j);
                if (g_beta) {
                    Basal<R> b = tau_basal(L.U(u, i, j), L.V(v, i, j - 1), L.V(v, i, j), L.V(v, i + 1, j - 1),
                                           L.V(v, i + 1, j), L.C(L.phi, i, j - 1), L.C(L.phi, i, j),
                                           L.C(L.beta, i, j - 1), L.C(L.beta, i, j), p.m, p.u_reg, p.water_drag);
                    if (j > 0) g_beta[i * nx + j - 1] += lul * b.d_beta0;
                    if (j < nx - 1) g_beta[i * nx + j] += lul * b.d_beta1;
                }
                if (g_bed) {
                    Driving<R> d = tau_driving(L.C(H, i, j - 1), L.C(H, i, j), L.C(L.bed, i, j - 1), L.C(L.bed, i, j),
                                               L.C(L.phi, i, j - 1), L.C(L.phi, i, j), dxi, j, nx);
                    if (j > 0) g_bed[i * nx + j - 1] += -lul * d.d_b0;
                    if (j < nx - 1) g_bed[i * nx + j] += -lul * d.d_b1;
                }
            }
            if (j < nx) {
                R lvt = L.V(lv, i, j);
                if (g_beta) {
                    Basal<R> b = tau_basal(L.V(v, i, j), L.U(u, i - 1, j), L.U(u, i - 1, j + 1), L.U(u, i, j),
                                           L.U(u, i, j + 1), L.C(L.phi, i - 1, j), L.C(L.phi, i, j),
                                           L.C(L.beta, i - 1, j), L.C(L.beta, i, j), p.m, p.u_reg, p.water_drag);
                    if (i > 0) g_beta[(i - 1) * nx + j] += lvt * b.d_beta0;
                    if (i < ny - 1) g_beta[i * nx + j] += lvt * b.d_beta1;
                }
                if (g_bed) {
                    Driving<R> d = tau_driving(L.C(H, i, j), L.C(H, i - 1, j), L.C(L.bed, i, j), L.C(L.bed, i - 1, j),
                                               L.C(L.phi, i, j), L.C(L.phi, i - 1, j), dxi, i, ny);
                    if (i > 0) g_bed[(i - 1) * nx + j] += -lvt * d.d_b1;
                    if (i < ny - 1) g_bed[i * nx + j] += -lvt * d.d_b0;
                }
            }
        }
}

// ---------------------------------------------------------------- transfers
// All restate glide/cuda/transfer.cu; coarse sizes (nyc, nxc), fine = 2x.
template <class R>
void restrict_u(const R* f, R* c, int nyc, int nxc) {  // transfer.cu:2-19
    for (int J = 0; J < nyc; ++J)
        for (int I = 0; I <= nxc; ++I)
            c[J * (nxc + 1) + I] = R(0.5) * (f[2 * J * (2 * nxc + 1) + 2 * I] + f[(2 * J + 1) * (2 * nxc + 1) + 2 * I]);
}
template <class R>
void restrict_v(const R* f, R* c, int nyc, int nxc) {  // transfer.cu:22-39
    for (int J = 0; J <= nyc; ++J)
        for (int I = 0; I < nxc; ++I)
            c[J * nxc + I] = R(0.5) * (f[2 * J * (2 * nxc) + 2 * I] + f[2 * J * (2 * nxc) + 2 * I + 1]);
}
template <class R>
void restrict_cell(const R* f, R* c, int nyc, int nxc, int how) {  // transfer.cu:42-139
    const int W = 2 * nxc;
    for (int J = 0; J < nyc; ++J)
        for (int I = 0; I < nxc; ++I) {
            R a = f[2 * J * W + 2 * I], b = f[2 * J * W + 2 * I + 1];
            R cc = f[(2 * J + 1) * W + 2 * I], d = f[(2 * J + 1) * W + 2 * I + 1];
            R o;
            if (how == 0) o = R(0.25) * (a + b + cc + d);
            else if (how == 1) o = std::max(std::max(a, b), std::max(cc, d));
            else if (how == 2) o = std::min(std::min(a, b), std::min(cc, d));
            else {
                R mu = R(0.25) * (a + b + cc + d);
                R d1 = a - mu, d2 = b - mu, d3 = cc - mu, d4 = d - mu;
                o = R(0.25) * (d1 * d1 + d2 * d2 + d3 * d3 + d4 * d4);
            }
            c[J * nxc + I] = o;
        }
}
// Bilinear interpolation of u-face data; also what the reference runs for
// v-face data (it launches this kernel on v arrays), so it takes the fine
// "u layout" sizes.  transfer.cu:177-229.
template <class R>
void prolong_u_bilinear(const R* c, R* f, int nyf, int nxf) {
    const int nyc = nyf / 2, nxc = nxf / 2;
    for (int idx = 0; idx < nyf * (nxf + 1); ++idx) {
        int j = idx / (nxf + 1), i = idx % (nxf + 1);
        R Jf = (R(j) - R(0.5)) * R(0.5), If = R(i) * R(0.5);
        Jf = std::max(R(0), std::min(Jf, R(nyc - 1)));
        If = std::max(R(0), std::min(If, R(nxc)));
        int Jlo = int(Jf), Ilo = int(If);
        int Jhi = std::min(Jlo + 1, nyc - 1), Ihi = std::min(Ilo + 1, nxc);
        R ty = Jf - R(Jlo), tx = If - R(Ilo);
        int s = nxc + 1;
        R v00 = c[Jlo * s + Ilo], v01 = c[Jlo * s + Ihi], v10 = c[Jhi * s + Ilo], v11 = c[Jhi * s + Ihi];
        f[idx] = (R(1) - ty) * ((R(1) - tx) * v00 + tx * v01) + ty * ((R(1) - tx) * v10 + tx * v11);
    }
}
template <class R>
void prolong_u_injection(const R* c, R* f, int nyf, int nxf) {  // transfer.cu:142-174
    for (int idx = 0; idx < nyf * (nxf + 1); ++idx) {
        int j = idx / (nxf + 1), i = idx % (nxf + 1);
        int J = j / 2, I = i / 2, s = nxf / 2 + 1;
        if (i % 2 == 0) f[idx] = c[J * s + I];
        else if (I < nxf / 2) f[idx] = R(0.5) * (c[J * s + I] + c[J * s + I + 1]);
        else f[idx] = c[J * s + I];
    }
}
template <class R>
void prolong_v_bilinear(const R* c, R* f, int nyf, int nxf) {  // transfer.cu:270-323
    const int nyc = nyf / 2, nxc = nxf / 2;
    for (int idx = 0; idx < (nyf + 1) * nxf; ++idx) {
        int j = idx / nxf, i = idx % nxf;
        R Jf = R(j) * R(0.5), If = (R(i) - R(0.5)) * R(0.5);
        Jf = std::max(R(0), std::min(Jf, R(nyc)));
        If = std::max(R(0), std::min(If, R(nxc - 1)));
        int Jlo = int(Jf), Ilo = int(If);
        int Jhi = std::min(Jlo + 1, nyc), Ihi = std::min(Ilo + 1, nxc - 1);
        R ty = Jf - R(Jlo), tx = If - R(Ilo);
        int s = nxc;
        R v00 = c[Jlo * s + Ilo], v01 = c[Jlo * s + Ihi], v10 = c[Jhi * s + Ilo], v11 = c[Jhi * s + Ihi];
        f[idx] = (R(1) - ty) * ((R(1) - tx) * v00 + tx * v01) + ty * ((R(1) - tx) * v10 + tx * v11);
    }
}
template <class R>
void prolong_v_injection(const R* c, R* f, int nyf, int nxf) {  // transfer.cu:232-267
    for (int idx = 0; idx < (nyf + 1) * nxf; ++idx) {
        int j = idx / nxf, i = idx % nxf;
        int J = j / 2, I = i / 2, s = nxf / 2;
        if (j % 2 == 0) f[idx] = c[J * s + I];
        else if (J < nyf / 2) f[idx] = R(0.5) * (c[J * s + I] + c[(J + 1) * s + I]);
        else f[idx] = c[J * s + I];
    }
}
template <class R>
void prolong_cell(const R* c, R* f, int nyf, int nxf, int bilinear) {  // transfer.cu:326-395
    const int nyc = nyf / 2, nxc = nxf / 2;
    for (int idx = 0; idx < nyf * nxf; ++idx) {
        int j = idx / nxf, i = idx % nxf;
        if (!bilinear) { f[idx] = c[(j / 2) * nxc + i / 2]; continue; }
        R Jf = (R(j) - R(0.5)) * R(0.5), If = (R(i) - R(0.5)) * R(0.5);
        Jf = std::max(R(0), std::min(Jf, R(nyc - 1)));
        If = std::max(R(0), std::min(If, R(nxc - 1)));
        int Jlo = int(Jf), Ilo = int(If);
        int Jhi = std::min(Jlo + 1, nyc - 1), Ihi = std::min(Ilo + 1, nxc - 1);
        R ty = Jf - R(Jlo), tx = If - R(Ilo);
        R v00 = c[Jlo * nxc + Ilo], v01 = c[Jlo * nxc + Ihi], v10 = c[Jhi * nxc + Ilo], v11 = c[Jhi * nxc + Ihi];
        f[idx] = (R(1) - ty) * ((R(1) - tx) * v00 + tx * v01) + ty * ((R(1) - tx) * v10 + tx * v11);
    }
}

}  // namespace oracle

// ------------------------------------------------------------- C interface
using namespace oracle;

#define GO_LEVEL_ARGS(R)                                                                    \
    int ny, int nx, const R *u, const R *v, const R *H, const R *phi, const R *mask,        \
        const R *f_u, const R *f_v, const R *f_H, const R *bed, const R *B, const R *beta,  \
        const R *gamma, const double *phys
#define GO_MAKE_LEVEL(R)                                                                    \
    Level<R> L{ny, nx, u, v, H, phi, mask, f_u, f_v, f_H, bed, B, beta, gamma};             \
    Phys<R> P{R(phys[0]), R(phys[1]), R(phys[2]), R(phys[3]), R(phys[4]), R(phys[5]),       \
              R(phys[6]), R(phys[7]), R(phys[8]), R(phys[9]), R(phys[10])};

#define GO_EXPORT(R, SUF)                                                                   \
    extern "C" void go_residual_##SUF(GO_LEVEL_ARGS(R), int use_forcing, int use_mask,      \
                                      R* r_u, R* r_v, R* r_H) {                             \
        GO_MAKE_LEVEL(R)                                                                    \
        residual(L, P, use_forcing != 0, use_mask != 0, r_u, r_v, r_H);                     \
    }                                                                                       \
    extern "C" void go_vanka_##SUF(GO_LEVEL_ARGS(R), int steps, double ssa_d, double mc_d,  \
                                   R* d_u, R* d_v, R* d_H, R* mask_out, int* iters) {       \
        GO_MAKE_LEVEL(R)                                                                    \
        vanka(L, P, NewtonCfg{steps, ssa_d, mc_d}, d_u, d_v, d_H, mask_out, iters);         \
    }                                                                                       \
    extern "C" void go_vanka_dump_##SUF(GO_LEVEL_ARGS(R), R* J, R* r) {                     \
        GO_MAKE_LEVEL(R)                                                                    \
        vanka_dump(L, P, J, r);                                                             \
    }                                                                                       \
    extern "C" void go_vjp_##SUF(GO_LEVEL_ARGS(R), const R* lu, const R* lv, const R* lH,   \
                                 int use_forcing, R* o_u, R* o_v, R* o_H) {                 \
        GO_MAKE_LEVEL(R)                                                                    \
        vjp(L, P, lu, lv, lH, use_forcing != 0, o_u, o_v, o_H);                             \
    }                                                                                       \
    extern "C" void go_vanka_adjoint_##SUF(GO_LEVEL_ARGS(R), double ssa_d, double mc_d,     \
                                           const R* ru, const R* rv, const R* rH, R* d_u,   \
                                           R* d_v, R* d_H) {                                \
        GO_MAKE_LEVEL(R)                                                                    \
        vanka_adjoint(L, P, ssa_d, mc_d, ru, rv, rH, d_u, d_v, d_H);                        \
    }                                                                                       \
    extern "C" void go_gradients_##SUF(GO_LEVEL_ARGS(R), const R* lu, const R* lv,          \
                                       R* g_beta, R* g_bed) {                               \
        GO_MAKE_LEVEL(R)                                                                    \
        gradients(L, P, lu, lv, g_beta, g_bed);                                             \
    }                                                                                       \
    extern "C" void go_grounded_##SUF(int ny, int nx, R* phi, const R* H, const R* bed,     \
                                      double c, double relax) {                             \
        compute_grounded(ny, nx, phi, H, bed, R(c), R(relax));                              \
    }                                                                                       \
    extern "C" void go_restrict_u_##SUF(const R* f, R* c, int nyc, int nxc) {               \
        restrict_u(f, c, nyc, nxc);                                                         \
    }                                                                                       \
    extern "C" void go_restrict_v_##SUF(const R* f, R* c, int nyc, int nxc) {               \
        restrict_v(f, c, nyc, nxc);                                                         \
    }                                                                                       \
    extern "C" void go_restrict_cell_##SUF(const R* f, R* c, int nyc, int nxc, int how) {   \
        restrict_cell(f, c, nyc, nxc, how);                                                 \
    }                                                                                       \
    extern "C" void go_prolong_u_##SUF(const R* c, R* f, int nyf, int nxf, int bilinear) {  \
        if (bilinear) prolong_u_bilinear(c, f, nyf, nxf);                                   \
        else prolong_u_injection(c, f, nyf, nxf);                                          \
    }                                                                                       \
    extern "C" void go_prolong_v_##SUF(const R* c, R* f, int nyf, int nxf, int bilinear) {  \
        if (bilinear) prolong_v_bilinear(c, f, nyf, nxf);                                   \
        else prolong_v_injection(c, f, nyf, nxf);                                          \
    }                                                                                       \
    extern "C" void go_prolong_cell_##SUF(const R* c, R* f, int nyf, int nxf, int bilinear) { \
        prolong_cell(c, f, nyf, nxf, bilinear);                                             \
    }

GO_EXPORT(double, f64)
GO_EXPORT(float, f32)
