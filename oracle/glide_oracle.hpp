// glide_oracle.hpp -- CPU restatement of the reference's discrete SSA + mass
// operator (TEST INFRASTRUCTURE: only tests/, smoke() and bench.py's CPU
// baseline leg may load it; the product never does).
//
// Everything here is written from the reference's published discretisation
// (JacobDowns/glide, glide/cuda/*.cu) in this project's own structure: plain
// loops over cells and faces, one function per physical term.  Each function
// cites the reference lines it restates.  Templated on the real type; the
// binary64 instantiation is the parity oracle for the FP64 CUDA path and the
// binary32 one is used for the mixed path.
//
// Index conventions (glide/grid.py:192-196, glide/cuda/common.cu:95-142):
//   cell (i, j): row i grows downward, column j; arrays (ny, nx) row-major
//   u(i, j)    : left face of cell (i, j);  array (ny, nx+1)
//   v(i, j)    : top face of cell (i, j);   array (ny+1, nx)
//   every read clamps its indices into the array (replicating edge values).
//
// Float literals that are not exact in binary32 (0.917f, 1e-6f) keep their
// binary32 value in every precision, as in the reference source.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle {

constexpr double kFlot = double(0.917f);     // rho_i / rho_w, common.cu:80, stress.cu:438
constexpr double kNewtonTol = double(1e-6f); // vanka.cu:540

template <class R>
struct Phys {
    R n, eps_reg, fr_driving, m, u_reg, water_drag, fr_sliding, calving_rate, fr_calving, dx, dt;
};

// One level's arrays (all contiguous row-major).
template <class R>
struct Level {
    int ny, nx;
    const R* u;      // (ny, nx+1)
    const R* v;      // (ny+1, nx)
    const R* H;      // (ny, nx)
    const R* phi;    // grounded fraction
    const R* mask;   // active-set mask
    const R* f_u;
    const R* f_v;
    const R* f_H;
    const R* bed;
    const R* B;
    const R* beta;
    const R* gamma;  // per-cell thickness floor

    static int cl(int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); }
    R U(const R* a, int i, int j) const { return a[cl(i, 0, ny - 1) * (nx + 1) + cl(j, 0, nx)]; }
    R V(const R* a, int i, int j) const { return a[cl(i, 0, ny) * nx + cl(j, 0, nx - 1)]; }
    R C(const R* a, int i, int j) const { return a[cl(i, 0, ny - 1) * nx + cl(j, 0, nx - 1)]; }
};

// ---------------------------------------------------------------- viscosity
// Cell viscosity eta = 1/2 B (eps_II + eps_reg)^((1-n)/(2n)), with the four
// corner shear rates zeroed where the corner lies on the domain edge.  The
// corner masks use the raw (unclamped) indices so that a cell outside the
// domain gets the same value the reference computes there.
// Restates viscosity.cu:119-168.
template <class R>
R eta_cell(const Level<R>& L, const R* u, const R* v, R n, R eps_reg, R dx, int i, int j) {
    const int ny = L.ny, nx = L.nx;
    R dxi = R(1) / dx;
    R gexp = (R(1) - n) / (R(2) * n);
    R ul = L.U(u, i, j), ur = L.U(u, i, j + 1), vt = L.V(v, i, j), vb = L.V(v, i + 1, j);
    R ux = (ur - ul) * dxi, vy = (vt - vb) * dxi;
    R m_tl = (i > 0 && j > 0), m_tr = (i > 0 && j < nx - 1);
    R m_bl = (i < ny - 1 && j > 0), m_br = (i < ny - 1 && j < nx - 1);
    R e_tl = R(0.5) * ((L.U(u, i - 1, j) - ul) * dxi + (vt - L.V(v, i, j - 1)) * dxi) * m_tl;
    R e_tr = R(0.5) * ((L.U(u, i - 1, j + 1) - ur) * dxi + (L.V(v, i, j + 1) - vt) * dxi) * m_tr;
    R e_bl = R(0.5) * ((ul - L.U(u, i + 1, j)) * dxi + (vb - L.V(v, i + 1, j - 1)) * dxi) * m_bl;
    R e_br = R(0.5) * ((ur - L.U(u, i + 1, j + 1)) * dxi + (L.V(v, i + 1, j + 1) - vb) * dxi) * m_br;
    R shear = R(0.25) * (e_tl * e_tl + e_tr * e_tr + e_bl * e_bl + e_br * e_br);
    R eII = ux * ux + vy * vy + ux * vy + shear + eps_reg;
    return R(0.5) * L.C(L.B, i, j) * std::pow(eII, gexp);
}

// Forward-mode derivative of eta_cell along (du, dv): returns d(eta).
// Restates the DualFloat overload, viscosity.cu:63-116.
template <class R>
R eta_cell_dot(const Level<R>& L, const R* u, const R* v, const R* du, const R* dv, R n,
               R eps_reg, R dx, int i, int j) {
    const int ny = L.ny, nx = L.nx;
    R dxi = R(1) / dx;
    R gexp = (R(1) - n) / (R(2) * n);
    R ul = L.U(u, i, j), ur = L.U(u, i, j + 1), vt = L.V(v, i, j), vb = L.V(v, i + 1, j);
    R dul = L.U(du, i, j), dur = L.U(du, i, j + 1), dvt = L.V(dv, i, j), dvb = L.V(dv, i + 1, j);
    R ux = (ur - ul) * dxi, vy = (vt - vb) * dxi;
    R dux = (dur - dul) * dxi, dvy = (dvt - dvb) * dxi;
    R m_tl = (i > 0 && j > 0), m_tr = (i > 0 && j < nx - 1);
    R m_bl = (i < ny - 1 && j > 0), m_br = (i < ny - 1 && j < nx - 1);
    auto corner = [&](R ua, R ub, R va, R vb2, R dua, R dub, R dva, R dvb2, R msk, R& e, R& de) {
        e = R(0.5) * ((ua - ub) * dxi + (va - vb2) * dxi) * msk;
        de = R(0.5) * ((dua - dub) * dxi + (dva - dvb2) * dxi) * msk;
    };
    R e1, d1, e2, d2, e3, d3, e4, d4;
    corner(L.U(u, i - 1, j), ul, vt, L.V(v, i, j - 1), L.U(du, i - 1, j), dul, dvt,
           L.V(dv, i, j - 1), m_tl, e1, d1);
    corner(L.U(u, i - 1, j + 1), ur, L.V(v, i, j + 1), vt, L.U(du, i - 1, j + 1), dur,
           L.V(dv, i, j + 1), dvt, m_tr, e2, d2);
    corner(ul, L.U(u, i + 1, j), vb, L.V(v, i + 1, j - 1), dul, L.U(du, i + 1, j), dvb,
           L.V(dv, i + 1, j - 1), m_bl, e3, d3);
    corner(ur, L.U(u, i + 1, j + 1), L.V(v, i + 1, j + 1), vb, dur, L.U(du, i + 1, j + 1),
           L.V(dv, i + 1, j + 1), dvb, m_br, e4, d4);
    R shear = R(0.25) * (e1 * e1 + e2 * e2 + e3 * e3 + e4 * e4);
    R dshear = R(0.25) * (R(2) * e1 * d1 + R(2) * e2 * d2 + R(2) * e3 * d3 + R(2) * e4 * d4);
    R eII = ux * ux + vy * vy + ux * vy + shear + eps_reg;
    R deII = R(2) * ux * dux + R(2) * vy * dvy + (ux * dvy + dux * vy) + dshear;
    return R(0.5) * L.C(L.B, i, j) * gexp * std::pow(eII, gexp - R(1)) * deII;
}

// Grounded fraction phi = sigmoid(c (bed + 0.917 H)), blended with the old
// value.  Restates common.cu:66-82 and viscosity.cu:17-36.
template <class R>
R grounded(R H, R bed, R c) {
    R z = bed + R(kFlot) * H;
    R s = std::min(std::max(c * z, R(-20)), R(20));
    return R(1) / (R(1) + std::exp(-s));
}

// ----------------------------------------------------------- stress terms
// Each term returns its value and the partial derivatives the residual,
// the local block Jacobian and the transpose need.
template <class R>
struct Normal { R s, d_ul, d_ur, d_vt, d_vb, d_etaH; };

// sigma_xx on cell (i, j) from its four faces and eta*H; zero off the domain
// in x.  Restates stress.cu:44-66.
template <class R>
Normal<R> sigma_xx(R ul, R ur, R vt, R vb, R etaH, R dxi, int j, int nx) {
    Normal<R> o{0, 0, 0, 0, 0, 0};
    if (j < 0 || j >= nx) return o;
    R exx = (R(2) * (ur - ul) * dxi + (vt - vb) * dxi);
    R p = R(2) * etaH * dxi;
    o.s = R(2) * etaH * exx;
    o.d_ul = -R(2) * p; o.d_ur = R(2) * p; o.d_vt = p; o.d_vb = -p; o.d_etaH = R(2) * exx;
    return o;
}

// sigma_yy on cell (i, j); zero off the domain in y.  Restates stress.cu:79-102.
template <class R>
Normal<R> sigma_yy(R ul, R ur, R vt, R vb, R etaH, R dxi, int i, int ny) {
    Normal<R> o{0, 0, 0, 0, 0, 0};
    if (i < 0 || i >= ny) return o;
    R eyy = ((ur - ul) * dxi + R(2) * (vt - vb) * dxi);
    R p = R(2) * etaH * dxi;
    o.s = R(2) * etaH * eyy;
    o.d_ul = -p; o.d_ur = p; o.d_vt = R(2) * p; o.d_vb = -R(2) * p; o.d_etaH = R(2) * eyy;
    return o;
}

template <class R>
struct Shear { R s, d_ut, d_ub, d_vl, d_vr, d_etaH; };

// sigma_xy on vertex (i, j) (top-left corner of cell (i, j)); zero on the
// domain boundary.  Restates stress.cu:160-183.
template <class R>
Shear<R> sigma_xy(R ut, R ub, R vl, R vr, R etaH, R dxi, int i, int j, int ny, int nx) {
    Shear<R> o{0, 0, 0, 0, 0, 0};
    if (i <= 0 || i >= ny || j <= 0 || j >= nx) return o;
    R exy = R(0.5) * ((ut - ub) * dxi + (vr - vl) * dxi);
    R p = etaH * dxi;
    o.s = R(2) * etaH * exy;
    o.d_ut = p; o.d_ub = -p; o.d_vl = -p; o.d_vr = p; o.d_etaH = R(2) * exy;
    return o;
}

// Vertex eta*H = mean over the four cells touching the vertex.
// Restates viscosity.cu:236-275.
template <class R>
R etaH_vertex(R e_tl, R e_tr, R e_bl, R e_br, R h_tl, R h_tr, R h_bl, R h_br) {
    return R(0.25) * (e_tl * h_tl + e_tr * h_tr + e_bl * h_bl + e_br * h_br);
}

template <class R>
struct Basal { R s, d_w, d_a, d_b, d_c, d_d, d_beta0, d_beta1; };

// Basal drag on a face: -(betā |u|^(m-1) + water_drag) w with
// betā = 1/2(beta0 phi0 + beta1 phi1) and |u|^2 = w^2 + 1/4 sum of the four
// tangential corner velocities squared.  Used for tau_bx (w = u, corners v)
// and tau_by (w = v, corners u).  The H-derivatives are identically zero.
// Restates stress.cu:254-279 and :342-369.
template <class R>
Basal<R> tau_basal(R w, R ca, R cb, R cc, R cd, R phi0, R phi1, R beta0, R beta1, R m,
                   R u_reg, R water_drag) {
    Basal<R> o;
    R be0 = beta0 * phi0, be1 = beta1 * phi1;
    R be = R(0.5) * (be0 + be1);
    R usq = w * w + R(0.25) * (ca * ca + cb * cb + cc * cc + cd * cd);
    R e = (m - R(1)) / R(2);
    R pw = std::pow(usq + u_reg, e);
    R dpw = e * std::pow(usq + u_reg, e - R(1));
    o.s = -(be * pw + water_drag) * w;
    o.d_w = -(be * (R(2) * dpw * w * w + pw) + water_drag);
    o.d_a = -be * (R(0.5) * dpw * w * ca);
    o.d_b = -be * (R(0.5) * dpw * w * cb);
    o.d_c = -be * (R(0.5) * dpw * w * cc);
    o.d_d = -be * (R(0.5) * dpw * w * cd);
    o.d_beta0 = -R(0.5) * phi0 * pw * w;
    o.d_beta1 = -R(0.5) * phi1 * pw * w;
    return o;
}

template <class R>
struct Driving { R s, d_H0, d_H1, d_b0, d_b1; };

// Driving stress on the face between cells 0 (left/bottom in index order is
// handled by the caller) and 1: H̄ (S1 - S0)/dx with
// S = phi b - (1 - phi) 0.917 H + H; zero on boundary faces.
// `lo`/`hi` are the face index and the number of cells along the axis.
// Restates stress.cu:419-454 (x) and :504-538 (y, with S_t - S_b).
template <class R>
Driving<R> tau_driving(R H0, R H1, R b0, R b1, R phi0, R phi1, R dxi, int k, int nk) {
    Driving<R> o{0, 0, 0, 0, 0};
    if (k <= 0 || k >= nk) return o;
    R Hm = R(0.5) * (H0 + H1);
    R base0 = phi0 * b0 - (R(1) - phi0) * R(kFlot) * H0;
    R base1 = phi1 * b1 - (R(1) - phi1) * R(kFlot) * H1;
    R db0 = -(R(1) - phi0) * R(kFlot);
    R db1 = -(R(1) - phi1) * R(kFlot);
    R S0 = base0 + H0, S1 = base1 + H1;
    o.s = Hm * (S1 - S0) * dxi;
    o.d_H0 = R(0.5) * (S1 - S0) * dxi - Hm * (R(1) + db0) * dxi;
    o.d_H1 = R(0.5) * (S1 - S0) * dxi + Hm * (R(1) + db1) * dxi;
    o.d_b0 = -Hm * phi0 * dxi;
    o.d_b1 = Hm * phi1 * dxi;
    return o;
}

template <class R>
struct Flux { R q, d_w, d_H0, d_H1; };

// Lax-Friedrichs mass flux through a face with normal velocity w between the
// cell before the face (H0) and after it (H1) in index order:
// q = H̄ w - 1/2 sqrt(w^2 + 10) (H1 - H0); zero on boundary faces.
// For y faces the reference orders the pair (top, bottom) with the sign of
// the jump reversed; the caller passes (H_b, H_t) so one formula serves both.
// Restates flux.cu:40-64 and :111-135.
template <class R>
Flux<R> lf_flux(R w, R H0, R H1, int k, int nk) {
    Flux<R> o{0, 0, 0, 0};
    if (k <= 0 || k >= nk) return o;
    R Hm = R(0.5) * (H0 + H1);
    R a = std::sqrt(w * w + R(10));
    R sgn = w / a;
    o.q = Hm * w - R(0.5) * a * (H1 - H0);
    o.d_H0 = R(0.5) * (w + a);
    o.d_H1 = R(0.5) * (w - a);
    o.d_w = Hm - R(0.5) * sgn * (H1 - H0);
    return o;
}

// Facet calving: (1 - phi_this)(1 - phi_other) c H_this.  Restates flux.cu:245-273.
template <class R>
R facet_calving(R H_this, R phi_this, R phi_other, R rate, R* d_H_this) {
    R coeff = (R(1) - phi_this) * (R(1) - phi_other);
    if (d_H_this) *d_H_this = coeff * rate;
    return coeff * rate * H_this;
}

}  // namespace oracle
