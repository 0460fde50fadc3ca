// stencil.cuh -- the discrete SSA momentum + mass operator on a staged tile.
//
// Device functions shared by the residual, Vanka and transpose kernels.  They
// evaluate the reference's discretisation (JacobDowns/glide glide/cuda/
// viscosity.cu, stress.cu, flux.cu) -- the same terms, sign conventions,
// boundary rules and evaluation order -- on values already staged in shared
// memory.  A stencil accessor `S` exposes, in global cell/face indices:
//   U(i,j) V(i,j)            face velocities (index-clamped at staging time)
//   Hc PHI BED BETA ETA(i,j) cell values
//   ny, nx                   level size
#pragma once

#include "glide_common.cuh"

namespace glide {

template <class R>
struct PhysR {
    R n, eps_reg, m, u_reg, water_drag, calving_rate, dx, dxi, dt, dti, gexp, c_ground;
    int glen3;  // n == 3: the viscosity power is a reciprocal cube root
    __device__ PhysR() {}
    __host__ __device__ PhysR(const Phys& p, double dx_, double dt_, double calving)
        : n(R(p.n)), eps_reg(R(p.eps_reg)), m(R(p.m)), u_reg(R(p.u_reg)),
          water_drag(R(p.water_drag)), calving_rate(R(calving)), dx(R(dx_)),
          dxi(R(1) / R(dx_)), dt(R(dt_)), dti(R(1) / R(dt_)), gexp((R(1) - R(p.n)) / (R(2) * R(p.n))),
          c_ground(R(p.fr_driving)), glen3(p.n == 3.0) {}
};

__device__ __forceinline__ double rcbrt_r(double x) { return rcbrt(x); }
__device__ __forceinline__ float rcbrt_r(float x) { return rcbrtf(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }

// x^((1-n)/(2n)); for Glen's n = 3 that is x^(-1/3), evaluated as a
// reciprocal cube root (a few ulp from pow, an order of magnitude cheaper).
template <class R>
__device__ __forceinline__ R glen_pow(R x, const PhysR<R>& p) {
    return p.glen3 ? rcbrt_r(x) : pow(x, p.gexp);
}

// x^((1-n)/(2n) - 1), the exponent of the viscosity's derivative.
template <class R>
__device__ __forceinline__ R glen_pow_m1(R x, const PhysR<R>& p) {
    if (p.glen3) {
        R r = rcbrt_r(x);
        R r2 = r * r;
        return r2 * r2;
    }
    return pow(x, p.gexp - R(1));
}

// Glen's-law cell viscosity from staged velocities; corner shear rates on
// the domain edge are masked with the raw indices (viscosity.cu:119-168).
template <class R, class S>
__device__ __forceinline__ R eta_at(const S& s, R Bc, const PhysR<R>& p, int i, int j) {
    const R dxi = p.dxi;
    const int ny = s.ny, nx = s.nx;
    R ul = s.U(i, j), ur = s.U(i, j + 1), vt = s.V(i, j), vb = s.V(i + 1, j);
    R ux = (ur - ul) * dxi, vy = (vt - vb) * dxi;
    R m_tl = (i > 0 && j > 0), m_tr = (i > 0 && j < nx - 1);
    R m_bl = (i < ny - 1 && j > 0), m_br = (i < ny - 1 && j < nx - 1);
    R e_tl = R(0.5) * ((s.U(i - 1, j) - ul) * dxi + (vt - s.V(i, j - 1)) * dxi) * m_tl;
    R e_tr = R(0.5) * ((s.U(i - 1, j + 1) - ur) * dxi + (s.V(i, j + 1) - vt) * dxi) * m_tr;
    R e_bl = R(0.5) * ((ul - s.U(i + 1, j)) * dxi + (vb - s.V(i + 1, j - 1)) * dxi) * m_bl;
    R e_br = R(0.5) * ((ur - s.U(i + 1, j + 1)) * dxi + (s.V(i + 1, j + 1) - vb) * dxi) * m_br;
    R shear = R(0.25) * (e_tl * e_tl + e_tr * e_tr + e_bl * e_bl + e_br * e_br);
    R eII = ux * ux + vy * vy + ux * vy + shear + p.eps_reg;
    return R(0.5) * Bc * glen_pow(eII, p);
}

// sigmoid grounding flag (common.cu:66-82)
template <class R>
__device__ __forceinline__ R grounded_frac(R H, R bed, R c) {
    R z = bed + R(kFlot) * H;
    R t = fmin(fmax(c * z, R(-20)), R(20));
    return R(1) / (R(1) + exp(-t));
}

template <class R>
struct NormalT { R s, d_ul, d_ur, d_vt, d_vb, d_eH; };
template <class R>
struct ShearT { R s, d_ut, d_ub, d_vl, d_vr, d_eH; };
template <class R>
struct BasalT { R s, d_w, d_a, d_b, d_c, d_d, d_b0, d_b1; };
template <class R>
struct DriveT { R s, d_H0, d_H1, d_b0, d_b1; };
template <class R>
struct FluxT { R q, d_w, d_H0, d_H1; };

// sigma_xx on cell column j (stress.cu:44-66)
template <class R>
__device__ __forceinline__ NormalT<R> sxx(R ul, R ur, R vt, R vb, R eH, R dxi, int j, int nx) {
    NormalT<R> o{0, 0, 0, 0, 0, 0};
    if (j < 0 || j >= nx) return o;
    R e = (R(2) * (ur - ul) * dxi + (vt - vb) * dxi);
    R q = R(2) * eH * dxi;
    o.s = R(2) * eH * e;
    o.d_ul = -R(2) * q; o.d_ur = R(2) * q; o.d_vt = q; o.d_vb = -q; o.d_eH = R(2) * e;
    return o;
}

// sigma_yy on cell row i (stress.cu:79-102)
template <class R>
__device__ __forceinline__ NormalT<R> syy(R ul, R ur, R vt, R vb, R eH, R dxi, int i, int ny) {
    NormalT<R> o{0, 0, 0, 0, 0, 0};
    if (i < 0 || i >= ny) return o;
    R e = ((ur - ul) * dxi + R(2) * (vt - vb) * dxi);
    R q = R(2) * eH * dxi;
    o.s = R(2) * eH * e;
    o.d_ul = -q; o.d_ur = q; o.d_vt = R(2) * q; o.d_vb = -R(2) * q; o.d_eH = R(2) * e;
    return o;
}

// sigma_xy on vertex (i, j), zero on the boundary (stress.cu:160-183)
template <class R>
__device__ __forceinline__ ShearT<R> sxy(R ut, R ub, R vl, R vr, R eH, R dxi, int i, int j, int ny, int nx) {
    ShearT<R> o{0, 0, 0, 0, 0, 0};
    if (i <= 0 || i >= ny || j <= 0 || j >= nx) return o;
    R e = R(0.5) * ((ut - ub) * dxi + (vr - vl) * dxi);
    R q = eH * dxi;
    o.s = R(2) * eH * e;
    o.d_ut = q; o.d_ub = -q; o.d_vl = -q; o.d_vr = q; o.d_eH = R(2) * e;
    return o;
}

template <class R>
__device__ __forceinline__ R vertex_eH(R e_tl, R e_tr, R e_bl, R e_br, R h_tl, R h_tr, R h_bl, R h_br) {
    return R(0.25) * (e_tl * h_tl + e_tr * h_tr + e_bl * h_bl + e_br * h_br);
}

// Weertman basal drag on a face (stress.cu:254-279, :342-369).  w is the
// face-normal velocity, a..d the four tangential corner velocities.
template <class R>
__device__ __forceinline__ BasalT<R> basal(R w, R a, R b, R c, R d, R ph0, R ph1, R be0, R be1,
                                           const PhysR<R>& p) {
    BasalT<R> o;
    R be = R(0.5) * (be0 * ph0 + be1 * ph1);
    R usq = w * w + R(0.25) * (a * a + b * b + c * c + d * d);
    R e = (p.m - R(1)) / R(2);
    R pw, dpw;
    if (e == R(0)) {  // linear sliding (m = 1): x^0 = 1 and 0 * x^-1 = +0 exactly
        pw = R(1);
        dpw = R(0);
    } else {
        pw = pow(usq + p.u_reg, e);
        dpw = e * pow(usq + p.u_reg, e - R(1));
    }
    o.s = -(be * pw + p.water_drag) * w;
    o.d_w = -(be * (R(2) * dpw * w * w + pw) + p.water_drag);
    o.d_a = -be * (R(0.5) * dpw * w * a);
    o.d_b = -be * (R(0.5) * dpw * w * b);
    o.d_c = -be * (R(0.5) * dpw * w * c);
    o.d_d = -be * (R(0.5) * dpw * w * d);
    o.d_b0 = -R(0.5) * ph0 * pw * w;
    o.d_b1 = -R(0.5) * ph1 * pw * w;
    return o;
}

// Driving stress H̄ (S1 - S0)/dx on the face between cells 0 and 1, zero on
// boundary faces (stress.cu:419-454, :504-538).
template <class R>
__device__ __forceinline__ DriveT<R> driving(R H0, R H1, R b0, R b1, R ph0, R ph1, R dxi, int k, int nk) {
    DriveT<R> o{0, 0, 0, 0, 0};
    if (k <= 0 || k >= nk) return o;
    R Hm = R(0.5) * (H0 + H1);
    R base0 = ph0 * b0 - (R(1) - ph0) * R(kFlot) * H0;
    R base1 = ph1 * b1 - (R(1) - ph1) * R(kFlot) * H1;
    R db0 = -(R(1) - ph0) * R(kFlot);
    R db1 = -(R(1) - ph1) * R(kFlot);
    R S0 = base0 + H0, S1 = base1 + H1;
    o.s = Hm * (S1 - S0) * dxi;
    o.d_H0 = R(0.5) * (S1 - S0) * dxi - Hm * (R(1) + db0) * dxi;
    o.d_H1 = R(0.5) * (S1 - S0) * dxi + Hm * (R(1) + db1) * dxi;
    o.d_b0 = -Hm * ph0 * dxi;
    o.d_b1 = Hm * ph1 * dxi;
    return o;
}

// Lax-Friedrichs mass flux between cells 0 and 1 in index order (for y faces
// the caller passes (bottom, top)), zero on boundary faces (flux.cu:40-64).
template <class R>
__device__ __forceinline__ FluxT<R> lflux(R w, R H0, R H1, int k, int nk) {
    FluxT<R> o{0, 0, 0, 0};
    if (k <= 0 || k >= nk) return o;
    R Hm = R(0.5) * (H0 + H1);
    const R q2 = w * w + R(10);
    const R ra = rsqrt_r(q2);
    R a = q2 * ra;   // sqrt(w^2 + 10)
    R sg = w * ra;   // w / sqrt(w^2 + 10)
    o.q = Hm * w - R(0.5) * a * (H1 - H0);
    o.d_H0 = R(0.5) * (w + a);
    o.d_H1 = R(0.5) * (w - a);
    o.d_w = Hm - R(0.5) * sg * (H1 - H0);
    return o;
}

// Facet calving flux (flux.cu:245-273)
template <class R>
__device__ __forceinline__ R calve(R Hthis, R ph_this, R ph_other, R rate, R& dH) {
    R c = (R(1) - ph_this) * (R(1) - ph_other);
    dH = c * rate;
    return c * rate * Hthis;
}

// ------------------------------------------------------------------ residual
// Mass residual of cell (i,j) before masking (residuals.cu:55-99)
template <class R, class S>
__device__ __forceinline__ R mass_residual(const S& s, const PhysR<R>& p, int i, int j, R fH) {
    const int ny = s.ny, nx = s.nx;
    const R dxi = p.dxi;
    R Hc = s.Hc(i, j), phc = s.PHI(i, j), dum;
    R r = Hc * p.dti;
    r -= fH;
    r -= lflux(s.U(i, j), s.Hc(i, j - 1), Hc, j, nx).q * dxi;
    r += calve(Hc, phc, s.PHI(i, j - 1), p.calving_rate, dum) * dxi;
    r += lflux(s.U(i, j + 1), Hc, s.Hc(i, j + 1), j + 1, nx).q * dxi;
    r += calve(Hc, phc, s.PHI(i, j + 1), p.calving_rate, dum) * dxi;
    r += lflux(s.V(i, j), Hc, s.Hc(i - 1, j), i, ny).q * dxi;
    r += calve(Hc, phc, s.PHI(i - 1, j), p.calving_rate, dum) * dxi;
    r -= lflux(s.V(i + 1, j), s.Hc(i + 1, j), Hc, i + 1, ny).q * dxi;
    r += calve(Hc, phc, s.PHI(i + 1, j), p.calving_rate, dum) * dxi;
    return r;
}

// x-momentum residual on u face (i,j) (residuals.cu:109-219)
template <class R, class S>
__device__ __forceinline__ R umom_residual(const S& s, const PhysR<R>& p, int i, int j, R fu) {
    const int ny = s.ny, nx = s.nx;
    const R dxi = p.dxi;
    R r = R(0) - fu;
    R Hc = s.Hc(i, j), Hl = s.Hc(i, j - 1), ul = s.U(i, j);
    r += sxx(ul, s.U(i, j + 1), s.V(i, j), s.V(i + 1, j), s.ETA(i, j) * Hc, dxi, j, nx).s * dxi;
    r -= sxx(s.U(i, j - 1), ul, s.V(i, j - 1), s.V(i + 1, j - 1), s.ETA(i, j - 1) * Hl, dxi, j - 1, nx).s * dxi;
    {
        R eH = vertex_eH(s.ETA(i - 1, j - 1), s.ETA(i - 1, j), s.ETA(i, j - 1), s.ETA(i, j),
                         s.Hc(i - 1, j - 1), s.Hc(i - 1, j), Hl, Hc);
        r += sxy(s.U(i - 1, j), ul, s.V(i, j - 1), s.V(i, j), eH, dxi, i, j, ny, nx).s * dxi;
    }
    {
        R eH = vertex_eH(s.ETA(i, j - 1), s.ETA(i, j), s.ETA(i + 1, j - 1), s.ETA(i + 1, j),
                         Hl, Hc, s.Hc(i + 1, j - 1), s.Hc(i + 1, j));
        r -= sxy(ul, s.U(i + 1, j), s.V(i + 1, j - 1), s.V(i + 1, j), eH, dxi, i + 1, j, ny, nx).s * dxi;
    }
    r += basal(ul, s.V(i, j - 1), s.V(i, j), s.V(i + 1, j - 1), s.V(i + 1, j), s.PHI(i, j - 1),
               s.PHI(i, j), s.BETA(i, j - 1), s.BETA(i, j), p).s;
    r -= driving(Hl, Hc, s.BED(i, j - 1), s.BED(i, j), s.PHI(i, j - 1), s.PHI(i, j), dxi, j, nx).s;
    if (j == 0 || j == nx) r = ul;
    return r;
}

// y-momentum residual on v face (i,j) (residuals.cu:221-331)
template <class R, class S>
__device__ __forceinline__ R vmom_residual(const S& s, const PhysR<R>& p, int i, int j, R fv) {
    const int ny = s.ny, nx = s.nx;
    const R dxi = p.dxi;
    R r = R(0) - fv;
    R Hc = s.Hc(i, j), Ht = s.Hc(i - 1, j), vt = s.V(i, j);
    r += syy(s.U(i - 1, j), s.U(i - 1, j + 1), s.V(i - 1, j), vt, s.ETA(i - 1, j) * Ht, dxi, i - 1, ny).s * dxi;
    r -= syy(s.U(i, j), s.U(i, j + 1), vt, s.V(i + 1, j), s.ETA(i, j) * Hc, dxi, i, ny).s * dxi;
    {
        R eH = vertex_eH(s.ETA(i - 1, j - 1), s.ETA(i - 1, j), s.ETA(i, j - 1), s.ETA(i, j),
                         s.Hc(i - 1, j - 1), Ht, s.Hc(i, j - 1), Hc);
        r -= sxy(s.U(i - 1, j), s.U(i, j), s.V(i, j - 1), vt, eH, dxi, i, j, ny, nx).s * dxi;
    }
    {
        R eH = vertex_eH(s.ETA(i - 1, j), s.ETA(i - 1, j + 1), s.ETA(i, j), s.ETA(i, j + 1),
                         Ht, s.Hc(i - 1, j + 1), Hc, s.Hc(i, j + 1));
        r += sxy(s.U(i - 1, j + 1), s.U(i, j + 1), vt, s.V(i, j + 1), eH, dxi, i, j + 1, ny, nx).s * dxi;
    }
    r += basal(vt, s.U(i - 1, j), s.U(i - 1, j + 1), s.U(i, j), s.U(i, j + 1), s.PHI(i - 1, j),
               s.PHI(i, j), s.BETA(i - 1, j), s.BETA(i, j), p).s;
    r -= driving(Hc, Ht, s.BED(i, j), s.BED(i - 1, j), s.PHI(i, j), s.PHI(i - 1, j), dxi, i, ny).s;
    if (i == 0 || i == ny) r = vt;
    return r;
}

// --------------------------------------------------------- local 5x5 system
// Newton matrix J (row-major) and residual r of the unknowns
// x = (u_l, u_r, v_t, v_b, H_c) of cell (i,j), neighbours and viscosity
// frozen (vanka.cu:91-475).
template <class R, class S>
__device__ __forceinline__ void local_system(const S& s, const PhysR<R>& p, int i, int j, const R* x,
                                             R* J, R* r) {
    const int ny = s.ny, nx = s.nx;
    const R dxi = p.dxi;
    const R ul = x[0], ur = x[1], vt = x[2], vb = x[3], Hc = x[4];
#pragma unroll
    for (int k = 0; k < 25; ++k) J[k] = R(0);
#pragma unroll
    for (int k = 0; k < 5; ++k) r[k] = R(0);
    const R phc = s.PHI(i, j), phl = s.PHI(i, j - 1), phr = s.PHI(i, j + 1);
    const R pht = s.PHI(i - 1, j), phb = s.PHI(i + 1, j);
    const R Hl = s.Hc(i, j - 1), Hr = s.Hc(i, j + 1), Ht = s.Hc(i - 1, j), Hb = s.Hc(i + 1, j);
    {
        R dc, c;
        J[24] = p.dti;
        r[4] += Hc * p.dti;
        FluxT<R> f = lflux(ul, Hl, Hc, j, nx);
        J[20] -= f.d_w * dxi; J[24] -= f.d_H1 * dxi; r[4] -= f.q * dxi;
        c = calve(Hc, phc, phl, p.calving_rate, dc); J[24] += dc * dxi; r[4] += c * dxi;
        f = lflux(ur, Hc, Hr, j + 1, nx);
        J[21] += f.d_w * dxi; J[24] += f.d_H0 * dxi; r[4] += f.q * dxi;
        c = calve(Hc, phc, phr, p.calving_rate, dc); J[24] += dc * dxi; r[4] += c * dxi;
        f = lflux(vt, Hc, Ht, i, ny);
        J[22] += f.d_w * dxi; J[24] += f.d_H0 * dxi; r[4] += f.q * dxi;
        c = calve(Hc, phc, pht, p.calving_rate, dc); J[24] += dc * dxi; r[4] += c * dxi;
        f = lflux(vb, Hb, Hc, i + 1, ny);
        J[23] -= f.d_w * dxi; J[24] -= f.d_H1 * dxi; r[4] -= f.q * dxi;
        c = calve(Hc, phc, phb, p.calving_rate, dc); J[24] += dc * dxi; r[4] += c * dxi;
    }
    const R ec = s.ETA(i, j);
    {
        NormalT<R> a = sxx(ul, ur, vt, vb, ec * Hc, dxi, j, nx);
        r[0] += a.s * dxi;
        J[0] += a.d_ul * dxi; J[1] += a.d_ur * dxi; J[2] += a.d_vt * dxi; J[3] += a.d_vb * dxi;
        J[4] += a.d_eH * ec * dxi;
        r[1] -= a.s * dxi;
        J[5] -= a.d_ul * dxi; J[6] -= a.d_ur * dxi; J[7] -= a.d_vt * dxi; J[8] -= a.d_vb * dxi;
        J[9] -= a.d_eH * ec * dxi;
        NormalT<R> b = syy(ul, ur, vt, vb, ec * Hc, dxi, i, ny);
        r[2] -= b.s * dxi;
        J[10] -= b.d_ul * dxi; J[11] -= b.d_ur * dxi; J[12] -= b.d_vt * dxi; J[13] -= b.d_vb * dxi;
        J[14] -= b.d_eH * ec * dxi;
        r[3] += b.s * dxi;
        J[15] += b.d_ul * dxi; J[16] += b.d_ur * dxi; J[17] += b.d_vt * dxi; J[18] += b.d_vb * dxi;
        J[19] += b.d_eH * ec * dxi;
    }
    {
        NormalT<R> a = sxx(s.U(i, j - 1), ul, s.V(i, j - 1), s.V(i + 1, j - 1), s.ETA(i, j - 1) * Hl, dxi, j - 1, nx);
        r[0] -= a.s * dxi; J[0] -= a.d_ur * dxi;
        a = sxx(ur, s.U(i, j + 2), s.V(i, j + 1), s.V(i + 1, j + 1), s.ETA(i, j + 1) * Hr, dxi, j + 1, nx);
        r[1] += a.s * dxi; J[6] += a.d_ul * dxi;
        a = syy(s.U(i - 1, j), s.U(i - 1, j + 1), s.V(i - 1, j), vt, s.ETA(i - 1, j) * Ht, dxi, i - 1, ny);
        r[2] += a.s * dxi; J[12] += a.d_vb * dxi;
        a = syy(s.U(i + 1, j), s.U(i + 1, j + 1), vb, s.V(i + 2, j), s.ETA(i + 1, j) * Hb, dxi, i + 1, ny);
        r[3] -= a.s * dxi; J[18] -= a.d_vt * dxi;
    }
    {
        const R q = R(0.25) * ec;
        R eH = vertex_eH(s.ETA(i - 1, j - 1), s.ETA(i - 1, j), s.ETA(i, j - 1), ec, s.Hc(i - 1, j - 1), Ht, Hl, Hc);
        ShearT<R> a = sxy(s.U(i - 1, j), ul, s.V(i, j - 1), vt, eH, dxi, i, j, ny, nx);
        r[0] += a.s * dxi; J[0] += a.d_ub * dxi; J[4] += a.d_eH * q * dxi;
        r[2] -= a.s * dxi; J[12] -= a.d_vr * dxi; J[14] -= a.d_eH * q * dxi;

        eH = vertex_eH(s.ETA(i - 1, j), s.ETA(i - 1, j + 1), ec, s.ETA(i, j + 1), Ht, s.Hc(i - 1, j + 1), Hc, Hr);
        a = sxy(s.U(i - 1, j + 1), ur, vt, s.V(i, j + 1), eH, dxi, i, j + 1, ny, nx);
        r[1] += a.s * dxi; J[6] += a.d_ub * dxi; J[9] += a.d_eH * q * dxi;
        r[2] += a.s * dxi; J[12] += a.d_vl * dxi; J[14] += a.d_eH * q * dxi;

        eH = vertex_eH(s.ETA(i, j - 1), ec, s.ETA(i + 1, j - 1), s.ETA(i + 1, j), Hl, Hc, s.Hc(i + 1, j - 1), Hb);
        a = sxy(ul, s.U(i + 1, j), s.V(i + 1, j - 1), vb, eH, dxi, i + 1, j, ny, nx);
        r[0] -= a.s * dxi; J[0] -= a.d_ut * dxi; J[4] -= a.d_eH * q * dxi;
        r[3] -= a.s * dxi; J[18] -= a.d_vr * dxi; J[19] -= a.d_eH * q * dxi;

        eH = vertex_eH(ec, s.ETA(i, j + 1), s.ETA(i + 1, j), s.ETA(i + 1, j + 1), Hc, Hr, Hb, s.Hc(i + 1, j + 1));
        a = sxy(ur, s.U(i + 1, j + 1), vb, s.V(i + 1, j + 1), eH, dxi, i + 1, j + 1, ny, nx);
        r[1] -= a.s * dxi; J[6] -= a.d_ut * dxi; J[9] -= a.d_eH * q * dxi;
        r[3] += a.s * dxi; J[18] += a.d_vl * dxi; J[19] += a.d_eH * q * dxi;
    }
    {
        const R bc = s.BETA(i, j);
        BasalT<R> b = basal(ul, s.V(i, j - 1), vt, s.V(i + 1, j - 1), vb, phl, phc, s.BETA(i, j - 1), bc, p);
        r[0] += b.s; J[0] += b.d_w; J[2] += b.d_b; J[3] += b.d_d;
        b = basal(ur, vt, s.V(i, j + 1), vb, s.V(i + 1, j + 1), phc, phr, bc, s.BETA(i, j + 1), p);
        r[1] += b.s; J[6] += b.d_w; J[7] += b.d_a; J[8] += b.d_c;
        b = basal(vt, s.U(i - 1, j), s.U(i - 1, j + 1), ul, ur, pht, phc, s.BETA(i - 1, j), bc, p);
        r[2] += b.s; J[12] += b.d_w; J[10] += b.d_c; J[11] += b.d_d;
        b = basal(vb, ul, ur, s.U(i + 1, j), s.U(i + 1, j + 1), phc, phb, bc, s.BETA(i + 1, j), p);
        r[3] += b.s; J[18] += b.d_w; J[15] += b.d_a; J[16] += b.d_b;
    }
    {
        const R bdc = s.BED(i, j);
        DriveT<R> d = driving(Hl, Hc, s.BED(i, j - 1), bdc, phl, phc, dxi, j, nx);
        r[0] -= d.s; J[4] -= d.d_H1;
        d = driving(Hc, Hr, bdc, s.BED(i, j + 1), phc, phr, dxi, j + 1, nx);
        r[1] -= d.s; J[9] -= d.d_H0;
        d = driving(Hc, Ht, bdc, s.BED(i - 1, j), phc, pht, dxi, i, ny);
        r[2] -= d.s; J[14] -= d.d_H0;
        d = driving(Hb, Hc, s.BED(i + 1, j), bdc, phb, phc, dxi, i + 1, ny);
        r[3] -= d.s; J[19] -= d.d_H1;
    }
}

template <class R>
__device__ __forceinline__ void pin(R* J, int k) {
#pragma unroll
    for (int c = 0; c < 5; ++c) J[k * 5 + c] = R(0);
#pragma unroll
    for (int a = 0; a < 5; ++a) J[a * 5 + k] = R(0);
    J[k * 5 + k] = R(1);
}

// In-place Doolittle LU without pivoting and the two triangular solves (the
// factorisation order of vanka.cu:5-48).  The pivot reciprocals computed by
// the factorisation are reused by the back substitution, so one reciprocal
// per pivot replaces the reference's extra divisions.  J is destroyed; b may
// alias x.
template <class R>
__device__ __forceinline__ void lu5_solve(R* J, const R* b, R* x) {
    R inv[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        inv[k] = R(1) / J[k * 5 + k];
#pragma unroll
        for (int a = k + 1; a < 5; ++a) {
            J[a * 5 + k] *= inv[k];
#pragma unroll
            for (int c = k + 1; c < 5; ++c) J[a * 5 + c] -= J[a * 5 + k] * J[k * 5 + c];
        }
    }
    R y0 = b[0];
    R y1 = b[1] - J[5] * y0;
    R y2 = b[2] - J[10] * y0 - J[11] * y1;
    R y3 = b[3] - J[15] * y0 - J[16] * y1 - J[17] * y2;
    R y4 = b[4] - J[20] * y0 - J[21] * y1 - J[22] * y2 - J[23] * y3;
    R x4 = y4 * inv[4];
    R x3 = (y3 - J[19] * x4) * inv[3];
    R x2 = (y2 - J[13] * x3 - J[14] * x4) * inv[2];
    R x1 = (y1 - J[7] * x2 - J[8] * x3 - J[9] * x4) * inv[1];
    R x0 = (y0 - J[1] * x1 - J[2] * x2 - J[3] * x3 - J[4] * x4) * inv[0];
    x[0] = x0; x[1] = x1; x[2] = x2; x[3] = x3; x[4] = x4;
}

}  // namespace glide
