// adjoint_kernels.cuh -- transpose of the coupled operator, adjoint block
// smoother and parameter gradients.
//
// The reference forms lambda^T dR/dx by scattering every residual row's
// partials onto the unknowns it touches with shared- and global-memory
// atomics (residuals.cu:667-1163).  Here each output entry GATHERS the same
// partials from the rows that touch it, in a fixed order: deterministic,
// atomic-free and owner-computes.  The per-row contributions are the
// reference's own (including its use of the forward derivative of eta along
// lambda for the viscous block, and its target filters: no contribution to
// the u faces on x = 0, nx, the v faces on y = 0, ny, or masked cells).
#pragma once

#include <cuda_bf16.h>

#include "forward_kernels.cuh"
#include "tma.cuh"

namespace glide {

constexpr int kTileA = 16;

// Forward derivative of the cell viscosity along (du, dv) (viscosity.cu:63-116).
template <class R, class S>
__device__ __forceinline__ R eta_dot_at(const S& s, R Bc, const PhysR<R>& p, int i, int j) {
    const R dxi = p.dxi;
    const int ny = s.ny, nx = s.nx;
    R ul = s.U(i, j), ur = s.U(i, j + 1), vt = s.V(i, j), vb = s.V(i + 1, j);
    R dul = s.LU(i, j), dur = s.LU(i, j + 1), dvt = s.LV(i, j), dvb = s.LV(i + 1, j);
    R ux = (ur - ul) * dxi, vy = (vt - vb) * dxi;
    R dux = (dur - dul) * dxi, dvy = (dvt - dvb) * dxi;
    R m_tl = (i > 0 && j > 0), m_tr = (i > 0 && j < nx - 1);
    R m_bl = (i < ny - 1 && j > 0), m_br = (i < ny - 1 && j < nx - 1);
    R e1 = R(0.5) * ((s.U(i - 1, j) - ul) * dxi + (vt - s.V(i, j - 1)) * dxi) * m_tl;
    R d1 = R(0.5) * ((s.LU(i - 1, j) - dul) * dxi + (dvt - s.LV(i, j - 1)) * dxi) * m_tl;
    R e2 = R(0.5) * ((s.U(i - 1, j + 1) - ur) * dxi + (s.V(i, j + 1) - vt) * dxi) * m_tr;
    R d2 = R(0.5) * ((s.LU(i - 1, j + 1) - dur) * dxi + (s.LV(i, j + 1) - dvt) * dxi) * m_tr;
    R e3 = R(0.5) * ((ul - s.U(i + 1, j)) * dxi + (vb - s.V(i + 1, j - 1)) * dxi) * m_bl;
    R d3 = R(0.5) * ((dul - s.LU(i + 1, j)) * dxi + (dvb - s.LV(i + 1, j - 1)) * dxi) * m_bl;
    R e4 = R(0.5) * ((ur - s.U(i + 1, j + 1)) * dxi + (s.V(i + 1, j + 1) - vb) * dxi) * m_br;
    R d4 = R(0.5) * ((dur - s.LU(i + 1, j + 1)) * dxi + (s.LV(i + 1, j + 1) - dvb) * dxi) * m_br;
    R shear = R(0.25) * (e1 * e1 + e2 * e2 + e3 * e3 + e4 * e4);
    R dshear = R(0.25) * (R(2) * e1 * d1 + R(2) * e2 * d2 + R(2) * e3 * d3 + R(2) * e4 * d4);
    R eII = ux * ux + vy * vy + ux * vy + shear + p.eps_reg;
    R deII = R(2) * ux * dux + R(2) * vy * dvy + (ux * dvy + dux * vy) + dshear;
    return R(0.5) * Bc * p.gexp * glen_pow_m1(eII, p) * deII;
}

// Staged tile for the transpose: forward state, lambda and B in box layout
// (TMA on large levels) with a two-cell halo -- u faces need rows
// [i0-3, i0+19), so the box starts at row i0 - 3 and is 24 rows high in
// binary32, 22 in binary64 (both multiples of 128 bytes) -- and eta, eta-dot
// on cells [i0-2, i0+18).
constexpr int kAdjBoxY = 3;
template <class R>
struct AdjTile {
    static constexpr int BH = sizeof(R) == 4 ? 24 : 22, NB = 9, NC = kTileA + 4, P = sizeof(R) == 4 ? 24 : NC;
    BoxT<R, BH> u, v, H, phi, bed, beta, B, lu, lv;  // staging order of the box maps
    R eta[NC][P], etad[NC][P];
};

template <class R>
struct AdjView {
    const AdjTile<R>& a;
    const Arr<R>* lH;
    const Arr<R>* mask;
    int i0, j0, ny, nx;
    static constexpr int A = 2;
    __device__ int r(int i) const { return i - (i0 - kAdjBoxY); }
    __device__ int c(int j) const { return j - (j0 - kBoxX); }
    __device__ R U(int i, int j) const { return a.u[r(i)][c(j)]; }
    __device__ R V(int i, int j) const { return a.v[r(i)][c(j)]; }
    __device__ R LU(int i, int j) const { return a.lu[r(i)][c(j)]; }
    __device__ R LV(int i, int j) const { return a.lv[r(i)][c(j)]; }
    __device__ R Hc(int i, int j) const { return a.H[r(i)][c(j)]; }
    __device__ R PHI(int i, int j) const { return a.phi[r(i)][c(j)]; }
    __device__ R BED(int i, int j) const { return a.bed[r(i)][c(j)]; }
    __device__ R BETA(int i, int j) const { return a.beta[r(i)][c(j)]; }
    __device__ R BC(int i, int j) const { return a.B[r(i)][c(j)]; }
    __device__ R ETA(int i, int j) const { return a.eta[i - (i0 - A)][j - (j0 - A)]; }
    __device__ R ETAD(int i, int j) const { return a.etad[i - (i0 - A)][j - (j0 - A)]; }
    // masked cell multiplier of a source cell inside the domain
    __device__ R LHm(int i, int j) const { return lH->at(i, j) * (R(1) - mask->at(i, j)); }
};

// Contributions of the mass row of cell (i,j) (residuals.cu:717-786).
template <class R>
struct CellSrc { R H0, Hl, Hr, Ht, Hb, Ul, Ur, Vt, Vb; };

template <class R, class S>
__device__ __forceinline__ CellSrc<R> cell_src(const S& s, const PhysR<R>& p, int i, int j, R fH) {
    const int ny = s.ny, nx = s.nx;
    const R dxi = p.dxi;
    CellSrc<R> o;
    R Hc = s.Hc(i, j), phc = s.PHI(i, j), dc;
    R lam = s.LHm(i, j);
    R h = lam * p.dti;
    FluxT<R> f = lflux(s.U(i, j), s.Hc(i, j - 1), Hc, j, nx);
    h += -lam * f.d_H1 * dxi; o.Hl = -lam * f.d_H0 * dxi; o.Ul = -lam * f.d_w * dxi;
    calve(Hc, phc, s.PHI(i, j - 1), p.calving_rate, dc); h += lam * dc * dxi;
    f = lflux(s.U(i, j + 1), Hc, s.Hc(i, j + 1), j + 1, nx);
    h += lam * f.d_H0 * dxi; o.Hr = lam * f.d_H1 * dxi; o.Ur = lam * f.d_w * dxi;
    calve(Hc, phc, s.PHI(i, j + 1), p.calving_rate, dc); h += lam * dc * dxi;
    f = lflux(s.V(i, j), Hc, s.Hc(i - 1, j), i, ny);
    h += lam * f.d_H0 * dxi; o.Ht = lam * f.d_H1 * dxi; o.Vt = lam * f.d_w * dxi;
    calve(Hc, phc, s.PHI(i - 1, j), p.calving_rate, dc); h += lam * dc * dxi;
    f = lflux(s.V(i + 1, j), s.Hc(i + 1, j), Hc, i + 1, ny);
    h += -lam * f.d_H1 * dxi; o.Hb = -lam * f.d_H0 * dxi; o.Vb = -lam * f.d_w * dxi;
    calve(Hc, phc, s.PHI(i + 1, j), p.calving_rate, dc); h += lam * dc * dxi;
    h += -fH;
    o.H0 = h;
    return o;
}

// Contributions of the x-momentum row on u face (i,j) (residuals.cu:791-936).
template <class R>
struct USrc { R U, H0, Hl, Htl, Ht, Hbl, Hb, Vtl, Vtr, Vbl, Vbr; };

template <class R, class S>
__device__ __forceinline__ USrc<R> u_src(const S& s, const PhysR<R>& p, int i, int j, R fu) {
    const int ny = s.ny, nx = s.nx;
    const R dxi = p.dxi;
    USrc<R> o;
    R Hc = s.Hc(i, j), Hl = s.Hc(i, j - 1), ul = s.U(i, j), lul = s.LU(i, j);
    R accU = 0, h0 = 0, hl = 0;
    {
        NormalT<R> a = sxx(ul, s.U(i, j + 1), s.V(i, j), s.V(i + 1, j), s.ETA(i, j) * Hc, dxi, j, nx);
        R t = a.d_ul * lul + a.d_ur * s.LU(i, j + 1) + a.d_vt * s.LV(i, j) + a.d_vb * s.LV(i + 1, j) +
              a.d_eH * (Hc * s.ETAD(i, j));
        accU += t * dxi;
        h0 += lul * a.d_eH * s.ETA(i, j) * dxi;
    }
    {
        NormalT<R> a = sxx(s.U(i, j - 1), ul, s.V(i, j - 1), s.V(i + 1, j - 1), s.ETA(i, j - 1) * Hl, dxi, j - 1, nx);
        R t = a.d_ul * s.LU(i, j - 1) + a.d_ur * lul + a.d_vt * s.LV(i, j - 1) + a.d_vb * s.LV(i + 1, j - 1) +
              a.d_eH * (Hl * s.ETAD(i, j - 1));
        accU += -t * dxi;
        hl += -lul * a.d_eH * s.ETA(i, j - 1) * dxi;
    }
    {
        R Htl = s.Hc(i - 1, j - 1), Ht = s.Hc(i - 1, j);
        R eH = vertex_eH(s.ETA(i - 1, j - 1), s.ETA(i - 1, j), s.ETA(i, j - 1), s.ETA(i, j), Htl, Ht, Hl, Hc);
        R deH = R(0.25) * Htl * s.ETAD(i - 1, j - 1) + R(0.25) * Ht * s.ETAD(i - 1, j) +
                R(0.25) * Hl * s.ETAD(i, j - 1) + R(0.25) * Hc * s.ETAD(i, j);
        ShearT<R> a = sxy(s.U(i - 1, j), ul, s.V(i, j - 1), s.V(i, j), eH, dxi, i, j, ny, nx);
        R t = a.d_ut * s.LU(i - 1, j) + a.d_ub * lul + a.d_vl * s.LV(i, j - 1) + a.d_vr * s.LV(i, j) + a.d_eH * deH;
        accU += t * dxi;
        R g = lul * a.d_eH;
        o.Htl = g * R(0.25) * s.ETA(i - 1, j - 1) * dxi;
        o.Ht = g * R(0.25) * s.ETA(i - 1, j) * dxi;
        hl += g * R(0.25) * s.ETA(i, j - 1) * dxi;
        h0 += g * R(0.25) * s.ETA(i, j) * dxi;
    }
    {
        R Hbl = s.Hc(i + 1, j - 1), Hb = s.Hc(i + 1, j);
        R eH = vertex_eH(s.ETA(i, j - 1), s.ETA(i, j), s.ETA(i + 1, j - 1), s.ETA(i + 1, j), Hl, Hc, Hbl, Hb);
        R deH = R(0.25) * Hl * s.ETAD(i, j - 1) + R(0.25) * Hc * s.ETAD(i, j) +
                R(0.25) * Hbl * s.ETAD(i + 1, j - 1) + R(0.25) * Hb * s.ETAD(i + 1, j);
        ShearT<R> a = sxy(ul, s.U(i + 1, j), s.V(i + 1, j - 1), s.V(i + 1, j), eH, dxi, i + 1, j, ny, nx);
        R t = a.d_ut * lul + a.d_ub * s.LU(i + 1, j) + a.d_vl * s.LV(i + 1, j - 1) + a.d_vr * s.LV(i + 1, j) +
              a.d_eH * deH;
        accU += -t * dxi;
        R g = lul * a.d_eH;
        hl += -g * R(0.25) * s.ETA(i, j - 1) * dxi;
        h0 += -g * R(0.25) * s.ETA(i, j) * dxi;
        o.Hbl = -g * R(0.25) * s.ETA(i + 1, j - 1) * dxi;
        o.Hb = -g * R(0.25) * s.ETA(i + 1, j) * dxi;
    }
    {
        BasalT<R> b = basal(ul, s.V(i, j - 1), s.V(i, j), s.V(i + 1, j - 1), s.V(i + 1, j), s.PHI(i, j - 1),
                            s.PHI(i, j), s.BETA(i, j - 1), s.BETA(i, j), p);
        accU += lul * b.d_w;
        o.Vtl = lul * b.d_a; o.Vtr = lul * b.d_b; o.Vbl = lul * b.d_c; o.Vbr = lul * b.d_d;
    }
    {
        DriveT<R> d = driving(Hl, Hc, s.BED(i, j - 1), s.BED(i, j), s.PHI(i, j - 1), s.PHI(i, j), dxi, j, nx);
        hl += -lul * d.d_H0;
        h0 += -lul * d.d_H1;
    }
    accU += -fu;
    o.U = accU; o.H0 = h0; o.Hl = hl;
    return o;
}

// Contributions of the y-momentum row on v face (i,j) (residuals.cu:938-1103).
template <class R>
struct VSrc { R V, Ht, H0, Htl, Hl, Htr, Hr, Utl, Utr, Ubl, Ubr; };

template <class R, class S>
__device__ __forceinline__ VSrc<R> v_src(const S& s, const PhysR<R>& p, int i, int j, R fv) {
    const int ny = s.ny, nx = s.nx;
    const R dxi = p.dxi;
    VSrc<R> o;
    R Hc = s.Hc(i, j), Ht = s.Hc(i - 1, j), vt = s.V(i, j), lvt = s.LV(i, j);
    R accV = 0, ht = 0, h0 = 0;
    {
        NormalT<R> a = syy(s.U(i - 1, j), s.U(i - 1, j + 1), s.V(i - 1, j), vt, s.ETA(i - 1, j) * Ht, dxi, i - 1, ny);
        R t = a.d_ul * s.LU(i - 1, j) + a.d_ur * s.LU(i - 1, j + 1) + a.d_vt * s.LV(i - 1, j) + a.d_vb * lvt +
              a.d_eH * (Ht * s.ETAD(i - 1, j));
        accV += t * dxi;
        ht += lvt * a.d_eH * s.ETA(i - 1, j) * dxi;
    }
    {
        NormalT<R> a = syy(s.U(i, j), s.U(i, j + 1), vt, s.V(i + 1, j), s.ETA(i, j) * Hc, dxi, i, ny);
        R t = a.d_ul * s.LU(i, j) + a.d_ur * s.LU(i, j + 1) + a.d_vt * lvt + a.d_vb * s.LV(i + 1, j) +
              a.d_eH * (Hc * s.ETAD(i, j));
        accV += -t * dxi;
        h0 += -lvt * a.d_eH * s.ETA(i, j) * dxi;
    }
    {
        R Htl = s.Hc(i - 1, j - 1), Hl = s.Hc(i, j - 1);
        R eH = vertex_eH(s.ETA(i - 1, j - 1), s.ETA(i - 1, j), s.ETA(i, j - 1), s.ETA(i, j), Htl, Ht, Hl, Hc);
        R deH = R(0.25) * Htl * s.ETAD(i - 1, j - 1) + R(0.25) * Ht * s.ETAD(i - 1, j) +
                R(0.25) * Hl * s.ETAD(i, j - 1) + R(0.25) * Hc * s.ETAD(i, j);
        ShearT<R> a = sxy(s.U(i - 1, j), s.U(i, j), s.V(i, j - 1), vt, eH, dxi, i, j, ny, nx);
        R t = a.d_ut * s.LU(i - 1, j) + a.d_ub * s.LU(i, j) + a.d_vl * s.LV(i, j - 1) + a.d_vr * lvt + a.d_eH * deH;
        accV += -t * dxi;
        R g = lvt * a.d_eH;
        o.Htl = -g * R(0.25) * s.ETA(i - 1, j - 1) * dxi;
        ht += -g * R(0.25) * s.ETA(i - 1, j) * dxi;
        o.Hl = -g * R(0.25) * s.ETA(i, j - 1) * dxi;
        h0 += -g * R(0.25) * s.ETA(i, j) * dxi;
    }
    {
        R Htr = s.Hc(i - 1, j + 1), Hr = s.Hc(i, j + 1);
        R eH = vertex_eH(s.ETA(i - 1, j), s.ETA(i - 1, j + 1), s.ETA(i, j), s.ETA(i, j + 1), Ht, Htr, Hc, Hr);
        R deH = R(0.25) * Ht * s.ETAD(i - 1, j) + R(0.25) * Htr * s.ETAD(i - 1, j + 1) +
                R(0.25) * Hc * s.ETAD(i, j) + R(0.25) * Hr * s.ETAD(i, j + 1);
        ShearT<R> a = sxy(s.U(i - 1, j + 1), s.U(i, j + 1), vt, s.V(i, j + 1), eH, dxi, i, j + 1, ny, nx);
        R t = a.d_ut * s.LU(i - 1, j + 1) + a.d_ub * s.LU(i, j + 1) + a.d_vl * lvt + a.d_vr * s.LV(i, j + 1) +
              a.d_eH * deH;
        accV += t * dxi;
        R g = lvt * a.d_eH;
        ht += g * R(0.25) * s.ETA(i - 1, j) * dxi;
        o.Htr = g * R(0.25) * s.ETA(i - 1, j + 1) * dxi;
        h0 += g * R(0.25) * s.ETA(i, j) * dxi;
        o.Hr = g * R(0.25) * s.ETA(i, j + 1) * dxi;
    }
    {
        BasalT<R> b = basal(vt, s.U(i - 1, j), s.U(i - 1, j + 1), s.U(i, j), s.U(i, j + 1), s.PHI(i - 1, j),
                            s.PHI(i, j), s.BETA(i - 1, j), s.BETA(i, j), p);
        accV += lvt * b.d_w;
        o.Utl = lvt * b.d_a; o.Utr = lvt * b.d_b; o.Ubl = lvt * b.d_c; o.Ubr = lvt * b.d_d;
    }
    {
        DriveT<R> d = driving(Hc, Ht, s.BED(i, j), s.BED(i - 1, j), s.PHI(i, j), s.PHI(i - 1, j), dxi, i, ny);
        ht += -lvt * d.d_H1;
        h0 += -lvt * d.d_H0;
    }
    accV += -fv;
    o.V = accV; o.Ht = ht; o.H0 = h0;
    return o;
}

template <class R>
struct VjpArgs {
    Arr<R> u, v, H, phi, mask, bed, B, beta;
    Arr<R> lu, lv, lH;
    Arr<R> f_u, f_v, f_H;   // forcing (use_forcing)
    Arr<R> o_u, o_v, o_H;   // outputs
    Arr<R> s_u, s_v, s_H;   // optional subtrahends
    double* partial;
    int* err;  // set when a bounded wait gives up
    PhysR<R> p;
    int ny, nx, use_forcing;
};

// Box maps in AdjTile staging order: u, v, H, phi, bed, beta, B, lambda_u,
// lambda_v.  Each warp computes a 4 x 8 patch of the 16 x 16 tile.
template <class R, class BLK>
__device__ __forceinline__ void vjp_tile(const VjpArgs<R>& a, const BoxMaps<9>& maps, BLK blk) {
    using TT = AdjTile<R>;
    constexpr int NC = TT::NC;
    __shared__ __align__(128) TT T;
    __shared__ double red[3][kTileA * kTileA / 32];
    __shared__ unsigned long long bar;
    const int i0 = blk.y() * kTileA, j0 = blk.x() * kTileA;
    const int ny = a.ny, nx = a.nx;
    {
        BoxT<R, TT::BH>* const dst[TT::NB] = {&T.u, &T.v, &T.H, &T.phi, &T.bed, &T.beta, &T.B, &T.lu, &T.lv};
        const Arr<R> src[TT::NB] = {a.u, a.v, a.H, a.phi, a.bed, a.beta, a.B, a.lu, a.lv};
        if (!stage_boxes<R, TT::NB, TT::BH, kAdjBoxY>(dst, src, maps, i0, j0, &bar, a.err)) return;
    }
    AdjView<R> s{T, &a.lH, &a.mask, i0, j0, ny, nx};
    for (int k = threadIdx.x; k < NC * NC; k += blockDim.x) {
        int r = k / NC, c = k % NC;
        int gi = i0 - 2 + r, gj = j0 - 2 + c;
        const R Bc = s.BC(gi, gj);
        T.eta[r][c] = eta_at<R>(s, Bc, a.p, gi, gj);
        T.etad[r][c] = eta_dot_at<R>(s, Bc, a.p, gi, gj);
    }
    __syncthreads();
    const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    const int I = i0 + 4 * (wp >> 1) + (ln >> 3), J = j0 + 8 * (wp & 1) + (ln & 7);
    double ssu = 0, ssv = 0, ssh = 0;
    const bool f = a.use_forcing != 0;
    const PhysR<R>& p = a.p;
    auto fu = [&](int i, int j) { return f ? a.f_u.at(i, j) : R(0); };
    auto fv = [&](int i, int j) { return f ? a.f_v.at(i, j) : R(0); };
    auto fh = [&](int i, int j) { return f ? a.f_H.at(i, j) : R(0); };
    if (I < ny && J < nx) {
        // Every residual row touching a target of this thread is evaluated
        // once; the target sums take fixed slots of those rows.
        const bool has_l = J > 0, has_r = J + 1 < nx, has_t = I > 0, has_b = I + 1 < ny;
        const CellSrc<R> c0 = cell_src(s, p, I, J, fh(I, J));
        const CellSrc<R> cl = has_l ? cell_src(s, p, I, J - 1, fh(I, J - 1)) : CellSrc<R>{};
        const CellSrc<R> ct = has_t ? cell_src(s, p, I - 1, J, fh(I - 1, J)) : CellSrc<R>{};
        const CellSrc<R> cr = has_r ? cell_src(s, p, I, J + 1, fh(I, J + 1)) : CellSrc<R>{};
        const CellSrc<R> cb = has_b ? cell_src(s, p, I + 1, J, fh(I + 1, J)) : CellSrc<R>{};
        const USrc<R> u0 = u_src(s, p, I, J, fu(I, J));
        const USrc<R> ur = u_src(s, p, I, J + 1, fu(I, J + 1));
        const USrc<R> utr = has_t ? u_src(s, p, I - 1, J + 1, fu(I - 1, J + 1)) : USrc<R>{};
        const USrc<R> ut = has_t ? u_src(s, p, I - 1, J, fu(I - 1, J)) : USrc<R>{};
        const USrc<R> ubr = has_b ? u_src(s, p, I + 1, J + 1, fu(I + 1, J + 1)) : USrc<R>{};
        const USrc<R> ub = has_b ? u_src(s, p, I + 1, J, fu(I + 1, J)) : USrc<R>{};
        const VSrc<R> v0 = v_src(s, p, I, J, fv(I, J));
        const VSrc<R> vb = v_src(s, p, I + 1, J, fv(I + 1, J));
        const VSrc<R> vbl = has_l ? v_src(s, p, I + 1, J - 1, fv(I + 1, J - 1)) : VSrc<R>{};
        const VSrc<R> vl = has_l ? v_src(s, p, I, J - 1, fv(I, J - 1)) : VSrc<R>{};
        const VSrc<R> vbr = has_r ? v_src(s, p, I + 1, J + 1, fv(I + 1, J + 1)) : VSrc<R>{};
        const VSrc<R> vr = has_r ? v_src(s, p, I, J + 1, fv(I, J + 1)) : VSrc<R>{};

        // u face (I, J): interior faces only
        R ou = 0;
        if (has_l) ou = c0.Ul + cl.Ur + u0.U + vb.Utl + vbl.Utr + v0.Ubl + vl.Ubr;
        if (a.s_u.p) ou = ou - a.s_u.at(I, J);
        a.o_u.at(I, J) = ou;
        ssu += double(ou) * double(ou);
        if (J == nx - 1) {
            R e = a.s_u.p ? R(0) - a.s_u.at(I, nx) : R(0);
            a.o_u.at(I, nx) = e;
            ssu += double(e) * double(e);
        }
        // v face (I, J): interior faces only
        R ov = 0;
        if (has_t) ov = c0.Vt + ct.Vb + v0.V + ur.Vtl + u0.Vtr + utr.Vbl + ut.Vbr;
        if (a.s_v.p) ov = ov - a.s_v.at(I, J);
        a.o_v.at(I, J) = ov;
        ssv += double(ov) * double(ov);
        if (I == ny - 1) {
            R e = a.s_v.p ? R(0) - a.s_v.at(ny, J) : R(0);
            a.o_v.at(ny, J) = e;
            ssv += double(e) * double(e);
        }
        // cell (I, J); masked cells receive nothing
        R oh = 0;
        if (!(a.mask.at(I, J) > R(0))) {
            oh = c0.H0;
            if (has_r) oh += cr.Hl;
            if (has_l) oh += cl.Hr;
            if (has_b) oh += cb.Ht;
            if (has_t) oh += ct.Hb;
            oh += u0.H0;
            oh += ur.Hl;
            if (has_b) oh += ubr.Htl + ub.Ht;
            if (has_t) oh += utr.Hbl + ut.Hb;
            oh += vb.Ht;
            oh += v0.H0;
            if (has_r) oh += vbr.Htl + vr.Hl;
            if (has_l) oh += vbl.Htr + vl.Hr;
        }
        if (a.s_H.p) oh = oh - a.s_H.at(I, J);
        a.o_H.at(I, J) = oh;
        ssh += double(oh) * double(oh);
    }
    if (a.partial) {
        for (int o = 16; o > 0; o >>= 1) {
            ssu += __shfl_down_sync(0xffffffffu, ssu, o);
            ssv += __shfl_down_sync(0xffffffffu, ssv, o);
            ssh += __shfl_down_sync(0xffffffffu, ssh, o);
        }
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l == 0) { red[0][w] = ssu; red[1][w] = ssv; red[2][w] = ssh; }
        __syncthreads();
        if (threadIdx.x < 3) {
            double acc = 0;
            for (int q = 0; q < kTileA * kTileA / 32; ++q) acc += red[threadIdx.x][q];
            a.partial[size_t(blk.y() * blk.gx() + blk.x()) * 3 + threadIdx.x] = acc;
        }
    }
}

template <class R>
__global__ void __launch_bounds__(kTileA * kTileA) k_vjp(VjpArgs<R> a,
                                                         const __grid_constant__ BoxMaps<9> maps) {
    vjp_tile<R>(a, maps, SoloBlock{});
}

// -------------------------------------------------------------------------
// Adjoint block smoother fused with the update lambda -= omega * delta
// (vanka.cu:663-797 plus glide/operators.py:517-524).  The local matrix is
// the forward one at the (fixed) forward state; the tile layout is the
// forward sweep's, so each block owns its faces and updates lambda in place.
// -------------------------------------------------------------------------
template <class R>
struct AdjSweepArgs {
    Arr<R> u, v, H, phi, mask, bed, B, beta;
    Arr<R> ru, rv, rH;     // adjoint residual
    Arr<R> lu, lv, lH;     // updated in place
    PhysR<R> p;
    R omega, ssa_damping, mc_damping;
    int ny, nx;
};

// TR = true: adjoint block smoother (solve with J^T; pinned rows get a zero
// right-hand side, as the reference does).  TR = false: the same smoother for
// the tangent system J e = f of the binary64 Newton outer iteration, whose
// pinned rows are identity rows (the correction there equals the residual).
template <class R, bool TR>
__global__ void __launch_bounds__(kSweepThreads) k_adjoint_sweep(AdjSweepArgs<R> a) {
    using TileT = Tile<R, kTile, 2, 1>;
    constexpr int NC = TileT::NC;
    constexpr int ND = kTile + 1;
    __shared__ TileT t;
    __shared__ R dl[ND][ND][4];
    const int i0 = blockIdx.y * kTile, j0 = blockIdx.x * kTile;
    const int ny = a.ny, nx = a.nx;
    stage_tile<R, kTile, 2, 1>(t, i0, j0, ny, nx, a.u, a.v, a.H, a.bed, a.beta, &a.phi);
    __syncthreads();
    TileView<R, kTile, 2, 1> s{t, i0, j0, ny, nx};
    for (int k = threadIdx.x; k < NC * NC; k += blockDim.x) {
        int r = k / NC, c = k % NC;
        int gi = i0 - 2 + r, gj = j0 - 2 + c;
        R Bc = a.B.at(clampi(gi, 0, ny - 1), clampi(gj, 0, nx - 1));
        t.eta[r][c] = eta_at<R>(s, Bc, a.p, gi, gj);
    }
    __syncthreads();
    int i, j;
    const int tid = threadIdx.x;
    if (tid < kTile * kTile) { i = i0 + tid / kTile; j = j0 + tid % kTile; }
    else if (tid < kTile * kTile + kTile) { i = i0 + (tid - kTile * kTile); j = j0 - 1; }
    else { i = i0 - 1; j = j0 + (tid - kTile * kTile - kTile); }
    const bool live = i >= 0 && i < ny && j >= 0 && j < nx;
    // the owned cells' unknowns, loaded with the factors rather than after the
    // barrier (only this thread writes them)
    const bool own = tid < kTile * kTile && live;
    R xu0 = R(0), xv0 = R(0), xh0 = R(0);
    if (own) {
        xu0 = a.xu.at(i, j);
        xv0 = a.xv.at(i, j);
        xh0 = a.xH.at(i, j);
    }
    R d4 = 0;
    R dd[4] = {0, 0, 0, 0};
    if (live) {
        R x[5] = {s.U(i, j), s.U(i, j + 1), s.V(i, j), s.V(i + 1, j), s.Hc(i, j)};
        R J[25], rr[5], JT[25], b[5], dlam[5];
        local_system<R>(s, a.p, i, j, x, J, rr);
        J[0] -= a.ssa_damping; J[6] -= a.ssa_damping; J[12] -= a.ssa_damping; J[18] -= a.ssa_damping;
        J[24] += a.mc_damping;
        b[0] = a.ru.at(i, j); b[1] = a.ru.at(i, j + 1); b[2] = a.rv.at(i, j); b[3] = a.rv.at(i + 1, j);
        b[4] = a.rH.at(i, j);
        const R zpin = R(0);
        if (j == 0) { pin(J, 0); b[0] = TR ? zpin : b[0]; }
        if (j == nx - 1) { pin(J, 1); b[1] = TR ? zpin : b[1]; }
        if (i == 0) { pin(J, 2); b[2] = TR ? zpin : b[2]; }
        if (i == ny - 1) { pin(J, 3); b[3] = TR ? zpin : b[3]; }
        if (a.mask.at(i, j) > R(0.5)) { pin(J, 4); b[4] = TR ? zpin : b[4]; }
        if (TR) {
#pragma unroll
            for (int r = 0; r < 5; ++r)
#pragma unroll
                for (int c = 0; c < 5; ++c) JT[r * 5 + c] = J[c * 5 + r];
            lu5_solve(JT, b, dlam);
        } else {
            lu5_solve(J, b, dlam);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) dd[q] = R(0.5) * dlam[q];
        d4 = dlam[4];
    }
    {
        const int di = i - (i0 - 1), dj = j - (j0 - 1);
#pragma unroll
        for (int q = 0; q < 4; ++q) dl[di][dj][q] = dd[q];
    }
    __syncthreads();
    if (tid < kTile * kTile && live) {
        const int di = i - (i0 - 1), dj = j - (j0 - 1);
        const R w = a.omega;
        R du = (j > 0 ? dl[di][dj - 1][1] : R(0)) + dl[di][dj][0];
        a.lu.at(i, j) = a.lu.at(i, j) - w * du;
        if (j == nx - 1) a.lu.at(i, nx) = a.lu.at(i, nx) - w * dl[di][dj][1];
        R dv = (i > 0 ? dl[di - 1][dj][3] : R(0)) + dl[di][dj][2];
        a.lv.at(i, j) = a.lv.at(i, j) - w * dv;
        if (i == ny - 1) a.lv.at(ny, j) = a.lv.at(ny, j) - w * dl[di][dj][3];
        a.lH.at(i, j) = a.lH.at(i, j) - w * d4;
    }
}

// -------------------------------------------------------------------------
// Block factors of the linear smoothers.  During a linear solve the state is
// fixed, so each cell's 5x5 block (local Newton matrix + damping, pinned
// rows, transposed for the adjoint) is factored once per V-cycle and stored:
// 25 values per cell, structure-of-arrays (value k of cell (i,j) at
// f[k * plane + i * pitch + j]), L below the diagonal, U above it and the
// pivot reciprocals on it.  The smoother then costs one triangular solve.
//
// The binary32 tangent smoother (the forward direction) stores its factors
// in bfloat16 pairs (8 significant bits, the binary32 exponent range) and
// solves with them in binary32: the stored factors are 25 of the 34 values a
// sweep moves per cell, and the smoother needs only an approximate inverse,
// since the Newton residual it serves covers every row.  The adjoint keeps
// binary32 factors: its sweep zeroes the pinned rows' right-hand side, so
// the values next to them are the smoother's own and would carry the
// factors' rounding into the converged adjoint.  Binary64 smoothers keep
// binary64 factors.  The buffer is sized for R either way.
// -------------------------------------------------------------------------
// Storage of one cell's 25 factors: kPlanes planes of `type`, at
// f[q * plane + i * pitch + j].
template <class R, bool TR>
struct FactorStore {
    using type = R;
    static constexpr int kPlanes = 25;
    static __device__ __forceinline__ void put(R* base, size_t plane, size_t at, const R (&M)[25]) {
        R* f = base + at;
#pragma unroll
        for (int k = 0; k < 25; ++k) f[k * plane] = M[k];
    }
    static __device__ __forceinline__ void get(const R* base, size_t plane, size_t at, R (&M)[25]) {
        const R* f = base + at;
#pragma unroll
        for (int k = 0; k < 25; ++k) M[k] = __ldg(f + k * plane);
    }
};
// bfloat16 pairs: factors 2q and 2q + 1 in plane q (factor 24 alone in plane
// 12), one 4-byte load per pair.
template <>
struct FactorStore<float, false> {
    using type = __nv_bfloat162;
    static constexpr int kPlanes = 13;
    static __device__ __forceinline__ void put(float* base, size_t plane, size_t at, const float (&M)[25]) {
        __nv_bfloat162* f = reinterpret_cast<__nv_bfloat162*>(base) + at;
#pragma unroll
        for (int q = 0; q < 13; ++q) f[q * plane] = __floats2bfloat162_rn(M[2 * q], q < 12 ? M[2 * q + 1] : 0.0f);
    }
    static __device__ __forceinline__ void get(const float* base, size_t plane, size_t at, float (&M)[25]) {
        const unsigned* f = reinterpret_cast<const unsigned*>(base) + at;
#pragma unroll
        for (int q = 0; q < 13; ++q) {
            const unsigned w = __ldg(f + q * plane);
            __nv_bfloat162 h;
            static_assert(sizeof(h) == sizeof(w), "a bfloat16 pair is one word");
            memcpy(&h, &w, sizeof(w));
            const float2 v = __bfloat1622float2(h);
            M[2 * q] = v.x;
            if (q < 12) M[2 * q + 1] = v.y;
        }
    }
};

template <class R>
struct BlockArgs {
    Arr<R> u, v, H, phi, mask, bed, B, beta;
    Arr<R> ru, rv, rH;  // residual of the linear system (sweep)
    Arr<R> xu, xv, xH;  // unknowns, updated in place (sweep)
    R* f;               // factors (FactorStore<R, TR> layout; the buffer holds 25 planes of R)
    size_t plane;
    int pitch;
    int* err;           // set when a bounded wait gives up
    PhysR<R> p;
    R omega, ssa_damping, mc_damping;
    int ny, nx;
};

template <class R, bool TR, class BLK>
__device__ __forceinline__ void block_factor_tile(const BlockArgs<R>& a, const BoxMaps<7>& maps, BLK blk) {
    using TileT = StateBoxTile<R>;
    constexpr int NC = TileT::NE;
    __shared__ __align__(128) TileT t;
    __shared__ unsigned long long bar;
    const int i0 = blk.y() * kTile, j0 = blk.x() * kTile;
    const int ny = a.ny, nx = a.nx;
    if (!stage_state_boxes<R>(t, maps, a.u, a.v, a.H, a.phi, a.bed, a.beta, a.B, i0, j0, &bar, a.err)) return;
    StateBoxView<R> s{t, i0, j0, ny, nx};
    for (int k = threadIdx.x; k < NC * NC; k += blockDim.x) {
        int r = k / NC, c = k % NC;
        int gi = i0 - 1 + r, gj = j0 - 1 + c;
        t.eta[r][c] = eta_at<R>(s, s.BC(gi, gj), a.p, gi, gj);
    }
    __syncthreads();
    const int i = i0 + threadIdx.x / kTile, j = j0 + threadIdx.x % kTile;
    if (i >= ny || j >= nx) return;
    R x[5] = {s.U(i, j), s.U(i, j + 1), s.V(i, j), s.V(i + 1, j), s.Hc(i, j)};
    R J[25], rr[5];
    local_system<R>(s, a.p, i, j, x, J, rr);
    J[0] -= a.ssa_damping; J[6] -= a.ssa_damping; J[12] -= a.ssa_damping; J[18] -= a.ssa_damping;
    J[24] += a.mc_damping;
    if (j == 0) pin(J, 0);
    if (j == nx - 1) pin(J, 1);
    if (i == 0) pin(J, 2);
    if (i == ny - 1) pin(J, 3);
    if (a.mask.at(i, j) > R(0.5)) pin(J, 4);
    R M[25];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int c = 0; c < 5; ++c) M[r * 5 + c] = TR ? J[c * 5 + r] : J[r * 5 + c];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const R inv = R(1) / M[k * 5 + k];
#pragma unroll
        for (int r = k + 1; r < 5; ++r) {
            M[r * 5 + k] *= inv;
#pragma unroll
            for (int c = k + 1; c < 5; ++c) M[r * 5 + c] -= M[r * 5 + k] * M[k * 5 + c];
        }
        M[k * 5 + k] = inv;
    }
    FactorStore<R, TR>::put(a.f, a.plane, size_t(i) * a.pitch + j, M);
}

template <class R, bool TR>
__global__ void __launch_bounds__(kTile * kTile)
    k_block_factor(BlockArgs<R> a, const __grid_constant__ BoxMaps<7> maps) {
    block_factor_tile<R, TR>(a, maps, SoloBlock{});
}

// One linear block-smoother sweep with stored factors: x += omega * delta
// with delta = B^-1 (f - Op x) per cell, face corrections averaged between
// the two cells of a face (adjoint: lambda -= omega * B^-T r, r = J^T lambda - f).
template <class R, bool TR, class BLK>
__device__ __forceinline__ void block_sweep_tile(const BlockArgs<R>& a, BLK blk) {
    constexpr int ND = kTile + 1;
    __shared__ R dl[ND][ND][4];
    const int i0 = blk.y() * kTile, j0 = blk.x() * kTile;
    const int ny = a.ny, nx = a.nx;
    int i, j;
    const int tid = threadIdx.x;
    if (tid < kTile * kTile) { i = i0 + tid / kTile; j = j0 + tid % kTile; }
    else if (tid < kTile * kTile + kTile) { i = i0 + (tid - kTile * kTile); j = j0 - 1; }
    else { i = i0 - 1; j = j0 + (tid - kTile * kTile - kTile); }
    const bool live = i >= 0 && i < ny && j >= 0 && j < nx;
    // the owned cells' unknowns, loaded with the factors rather than after the
    // barrier (only this thread writes them)
    const bool own = tid < kTile * kTile && live;
    R xu0 = R(0), xv0 = R(0), xh0 = R(0);
    if (own) {
        xu0 = a.xu.at(i, j);
        xv0 = a.xv.at(i, j);
        xh0 = a.xH.at(i, j);
    }
    R d4 = 0;
    R dd[4] = {0, 0, 0, 0};
    if (live) {
        R b[5] = {a.ru.at(i, j), a.ru.at(i, j + 1), a.rv.at(i, j), a.rv.at(i + 1, j), a.rH.at(i, j)};
        if (TR) {  // the adjoint zeroes the pinned rows' right-hand side
            if (j == 0) b[0] = R(0);
            if (j == nx - 1) b[1] = R(0);
            if (i == 0) b[2] = R(0);
            if (i == ny - 1) b[3] = R(0);
            if (a.mask.at(i, j) > R(0.5)) b[4] = R(0);
        }
        R M[25];
        FactorStore<R, TR>::get(a.f, a.plane, size_t(i) * a.pitch + j, M);
        R y0 = b[0];
        R y1 = b[1] - M[5] * y0;
        R y2 = b[2] - M[10] * y0 - M[11] * y1;
        R y3 = b[3] - M[15] * y0 - M[16] * y1 - M[17] * y2;
        R y4 = b[4] - M[20] * y0 - M[21] * y1 - M[22] * y2 - M[23] * y3;
        R x4 = y4 * M[24];
        R x3 = (y3 - M[19] * x4) * M[18];
        R x2 = (y2 - M[13] * x3 - M[14] * x4) * M[12];
        R x1 = (y1 - M[7] * x2 - M[8] * x3 - M[9] * x4) * M[6];
        R x0 = (y0 - M[1] * x1 - M[2] * x2 - M[3] * x3 - M[4] * x4) * M[0];
        dd[0] = R(0.5) * x0; dd[1] = R(0.5) * x1; dd[2] = R(0.5) * x2; dd[3] = R(0.5) * x3;
        d4 = x4;
    }
    {
        const int di = i - (i0 - 1), dj = j - (j0 - 1);
#pragma unroll
        for (int q = 0; q < 4; ++q) dl[di][dj][q] = dd[q];
    }
    __syncthreads();
    if (own) {
        const int di = i - (i0 - 1), dj = j - (j0 - 1);
        const R w = a.omega;
        R du = (j > 0 ? dl[di][dj - 1][1] : R(0)) + dl[di][dj][0];
        a.xu.at(i, j) = xu0 - w * du;
        if (j == nx - 1) a.xu.at(i, nx) = a.xu.at(i, nx) - w * dl[di][dj][1];
        R dv = (i > 0 ? dl[di - 1][dj][3] : R(0)) + dl[di][dj][2];
        a.xv.at(i, j) = xv0 - w * dv;
        if (i == ny - 1) a.xv.at(ny, j) = a.xv.at(ny, j) - w * dl[di][dj][3];
        a.xH.at(i, j) = xh0 - w * d4;
    }
}

template <class R, bool TR>
__global__ void __launch_bounds__(kSweepThreads) k_block_sweep(BlockArgs<R> a) {
    block_sweep_tile<R, TR>(a, SoloBlock{});
}

// -------------------------------------------------------------------------
// Gradients (grad.cu:2-169, glide/operators.py:589-593), gathered per cell
// with the reference's index guards.
// -------------------------------------------------------------------------
template <class R>
struct GradArgs {
    Arr<R> u, v, H, phi, bed, beta;
    Arr<R> lu, lv, lH;
    Arr<R> g_beta, g_bed, g_Hp, g_smb;
    PhysR<R> p;
    R dt;
    int ny, nx;
};

template <class R>
struct GView {
    const GradArgs<R>& a;
    int ny, nx;
    __device__ R U(int i, int j) const { return a.u.at(clampi(i, 0, ny - 1), clampi(j, 0, nx)); }
    __device__ R V(int i, int j) const { return a.v.at(clampi(i, 0, ny), clampi(j, 0, nx - 1)); }
    __device__ R C(const Arr<R>& f, int i, int j) const { return f.at(clampi(i, 0, ny - 1), clampi(j, 0, nx - 1)); }
};

template <class R>
__device__ __forceinline__ void gradients_at(const GradArgs<R>& a, int I, int J) {
    const int ny = a.ny, nx = a.nx;
    if (J >= nx) return;
    GView<R> g{a, ny, nx};
    const R dxi = a.p.dxi;
    // basal drag / driving stress of u face (i, j)
    auto ub = [&](int i, int j) {
        return basal(g.U(i, j), g.V(i, j - 1), g.V(i, j), g.V(i + 1, j - 1), g.V(i + 1, j), g.C(a.phi, i, j - 1),
                     g.C(a.phi, i, j), g.C(a.beta, i, j - 1), g.C(a.beta, i, j), a.p);
    };
    auto ud = [&](int i, int j) {
        return driving(g.C(a.H, i, j - 1), g.C(a.H, i, j), g.C(a.bed, i, j - 1), g.C(a.bed, i, j),
                       g.C(a.phi, i, j - 1), g.C(a.phi, i, j), dxi, j, nx);
    };
    auto vb = [&](int i, int j) {
        return basal(g.V(i, j), g.U(i - 1, j), g.U(i - 1, j + 1), g.U(i, j), g.U(i, j + 1), g.C(a.phi, i - 1, j),
                     g.C(a.phi, i, j), g.C(a.beta, i - 1, j), g.C(a.beta, i, j), a.p);
    };
    auto vd = [&](int i, int j) {
        return driving(g.C(a.H, i, j), g.C(a.H, i - 1, j), g.C(a.bed, i, j), g.C(a.bed, i - 1, j),
                       g.C(a.phi, i, j), g.C(a.phi, i - 1, j), dxi, i, ny);
    };
    if (a.g_beta.p) {
        R s = a.lu.at(I, J + 1) * ub(I, J + 1).d_b0;
        if (J < nx - 1) s += a.lu.at(I, J) * ub(I, J).d_b1;
        s += a.lv.at(I + 1, J) * vb(I + 1, J).d_b0;
        if (I < ny - 1) s += a.lv.at(I, J) * vb(I, J).d_b1;
        a.g_beta.at(I, J) = s;
    }
    if (a.g_bed.p) {
        R s = -a.lu.at(I, J + 1) * ud(I, J + 1).d_b0;
        if (J < nx - 1) s += -a.lu.at(I, J) * ud(I, J).d_b1;
        s += -a.lv.at(I + 1, J) * vd(I + 1, J).d_b1;
        if (I < ny - 1) s += -a.lv.at(I, J) * vd(I, J).d_b0;
        a.g_bed.at(I, J) = s;
    }
    if (a.g_Hp.p) a.g_Hp.at(I, J) = -a.lH.at(I, J) / a.dt;
    if (a.g_smb.p) a.g_smb.at(I, J) = -a.lH.at(I, J);
}

template <class R>
__global__ void k_gradients(GradArgs<R> a) {
    gradients_at(a, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

}  // namespace glide
