// tangent_kernels.cuh -- Jacobian-vector product of the coupled operator.
//
// r_lin = J(x) e - f over one level: the exact directional derivative of the
// residual rows along e = (e_u, e_v, e_H), the grounded fraction held fixed
// (as the reference's forward-mode kernel does, residuals.cu:341-660), with
// the rows the solver pins written as identity rows: Dirichlet faces
// (u on x = 0, nx; v on y = 0, ny) and active-set cells (mask = 1) give
// r_lin = e - f there.  With `ref_rows` the pinned rows follow the reference
// kernel instead (zero on Dirichlet faces, (1 - mask) times the mass row).
#pragma once

#include "adjoint_kernels.cuh"
#include "tma.cuh"

namespace glide {

// d(mass row of cell (i,j)) . e before masking (residuals.cu:391-439)
template <class R, class S>
__device__ __forceinline__ R mass_jvp(const S& s, const PhysR<R>& p, int i, int j) {
    const int ny = s.ny, nx = s.nx;
    const R dxi = p.dxi;
    const R Hc = s.Hc(i, j), phc = s.PHI(i, j), eHc = s.EH(i, j);
    R dc, d = eHc * p.dti;
    FluxT<R> f = lflux(s.U(i, j), s.Hc(i, j - 1), Hc, j, nx);
    d -= (f.d_w * s.LU(i, j) + f.d_H0 * s.EH(i, j - 1) + f.d_H1 * eHc) * dxi;
    calve(Hc, phc, s.PHI(i, j - 1), p.calving_rate, dc); d += dc * eHc * dxi;
    f = lflux(s.U(i, j + 1), Hc, s.Hc(i, j + 1), j + 1, nx);
    d += (f.d_w * s.LU(i, j + 1) + f.d_H0 * eHc + f.d_H1 * s.EH(i, j + 1)) * dxi;
    calve(Hc, phc, s.PHI(i, j + 1), p.calving_rate, dc); d += dc * eHc * dxi;
    f = lflux(s.V(i, j), Hc, s.Hc(i - 1, j), i, ny);
    d += (f.d_w * s.LV(i, j) + f.d_H0 * eHc + f.d_H1 * s.EH(i - 1, j)) * dxi;
    calve(Hc, phc, s.PHI(i - 1, j), p.calving_rate, dc); d += dc * eHc * dxi;
    f = lflux(s.V(i + 1, j), s.Hc(i + 1, j), Hc, i + 1, ny);
    d -= (f.d_w * s.LV(i + 1, j) + f.d_H0 * s.EH(i + 1, j) + f.d_H1 * eHc) * dxi;
    calve(Hc, phc, s.PHI(i + 1, j), p.calving_rate, dc); d += dc * eHc * dxi;
    return d;
}

// Linearised stresses along e, built from the per-cell products the tile
// holds: etaH = eta H and detaH = eta-dot H + eta e_H (the derivative of
// eta H).  Each is the stress routine's derivative coefficients (stress.cu;
// sxx / syy / sxy in stencil.cuh) contracted with e.
//
// sigma_xx H on cell (i, j) (stress.cu:44-66): d_ul = -2q, d_ur = 2q,
// d_vt = q, d_vb = -q with q = 2 eta H dxi, d_eH = 2 e.
template <class R, class S>
__device__ __forceinline__ R nxx_lin(const S& s, R dxi, int i, int j, int nx) {
    if (j < 0 || j >= nx) return R(0);
    const R e = R(2) * (s.U(i, j + 1) - s.U(i, j)) * dxi + (s.V(i, j) - s.V(i + 1, j)) * dxi;
    const R q = R(2) * s.ETAH(i, j) * dxi;
    return q * (R(2) * (s.LU(i, j + 1) - s.LU(i, j)) + (s.LV(i, j) - s.LV(i + 1, j))) + R(2) * e * s.DETAH(i, j);
}

// sigma_yy H on cell (i, j) (stress.cu:79-102): d_ul = -q, d_ur = q,
// d_vt = 2q, d_vb = -2q, d_eH = 2 e.
template <class R, class S>
__device__ __forceinline__ R nyy_lin(const S& s, R dxi, int i, int j, int ny) {
    if (i < 0 || i >= ny) return R(0);
    const R e = (s.U(i, j + 1) - s.U(i, j)) * dxi + R(2) * (s.V(i, j) - s.V(i + 1, j)) * dxi;
    const R q = R(2) * s.ETAH(i, j) * dxi;
    return q * ((s.LU(i, j + 1) - s.LU(i, j)) + R(2) * (s.LV(i, j) - s.LV(i + 1, j))) + R(2) * e * s.DETAH(i, j);
}

// sigma_xy H on vertex (i, j), zero on the boundary (stress.cu:160-183), with
// the vertex's eta H the mean of its four cells: d_ut = q, d_ub = -q,
// d_vl = -q, d_vr = q with q = eta H dxi, d_eH = 2 e.
template <class R, class S>
__device__ __forceinline__ R sxy_lin(const S& s, R dxi, int i, int j, int ny, int nx) {
    if (i <= 0 || i >= ny || j <= 0 || j >= nx) return R(0);
    const R e = R(0.5) * ((s.U(i - 1, j) - s.U(i, j)) * dxi + (s.V(i, j) - s.V(i, j - 1)) * dxi);
    const R eH = R(0.25) * (s.ETAH(i - 1, j - 1) + s.ETAH(i - 1, j) + s.ETAH(i, j - 1) + s.ETAH(i, j));
    const R deH = R(0.25) * (s.DETAH(i - 1, j - 1) + s.DETAH(i - 1, j) + s.DETAH(i, j - 1) + s.DETAH(i, j));
    const R q = eH * dxi;
    return q * ((s.LU(i - 1, j) - s.LU(i, j)) + (s.LV(i, j) - s.LV(i, j - 1))) + R(2) * e * deH;
}

// d(x-momentum row on u face (i,j)) . e and d(y-momentum row on v face
// (i,j)) . e for interior rows (residuals.cu:441-658).  The shear on vertex
// (i, j) enters both rows and is evaluated once; `want_u` / `want_v` skip a
// row the caller pins.
template <class R, class S>
__device__ __forceinline__ void mom_jvp(const S& s, const PhysR<R>& p, int i, int j, bool want_u, bool want_v,
                                        R& du, R& dv) {
    const int ny = s.ny, nx = s.nx;
    const R dxi = p.dxi;
    const R sh = sxy_lin<R>(s, dxi, i, j, ny, nx);
    if (want_u) {
        const R Hc = s.Hc(i, j), Hl = s.Hc(i, j - 1), ul = s.U(i, j);
        R d = 0;
        d += nxx_lin<R>(s, dxi, i, j, nx) * dxi;
        d -= nxx_lin<R>(s, dxi, i, j - 1, nx) * dxi;
        d += sh * dxi;
        d -= sxy_lin<R>(s, dxi, i + 1, j, ny, nx) * dxi;
        {
            BasalT<R> b = basal(ul, s.V(i, j - 1), s.V(i, j), s.V(i + 1, j - 1), s.V(i + 1, j), s.PHI(i, j - 1),
                                s.PHI(i, j), s.BETA(i, j - 1), s.BETA(i, j), p);
            d += b.d_w * s.LU(i, j) + b.d_a * s.LV(i, j - 1) + b.d_b * s.LV(i, j) + b.d_c * s.LV(i + 1, j - 1) +
                 b.d_d * s.LV(i + 1, j);
        }
        {
            DriveT<R> dr = driving(Hl, Hc, s.BED(i, j - 1), s.BED(i, j), s.PHI(i, j - 1), s.PHI(i, j), dxi, j, nx);
            d -= dr.d_H0 * s.EH(i, j - 1) + dr.d_H1 * s.EH(i, j);
        }
        du = d;
    }
    if (want_v) {
        const R Hc = s.Hc(i, j), Ht = s.Hc(i - 1, j), vt = s.V(i, j);
        R d = 0;
        d += nyy_lin<R>(s, dxi, i - 1, j, ny) * dxi;
        d -= nyy_lin<R>(s, dxi, i, j, ny) * dxi;
        d -= sh * dxi;
        d += sxy_lin<R>(s, dxi, i, j + 1, ny, nx) * dxi;
        {
            BasalT<R> b = basal(vt, s.U(i - 1, j), s.U(i - 1, j + 1), s.U(i, j), s.U(i, j + 1), s.PHI(i - 1, j),
                                s.PHI(i, j), s.BETA(i - 1, j), s.BETA(i, j), p);
            d += b.d_w * s.LV(i, j) + b.d_a * s.LU(i - 1, j) + b.d_b * s.LU(i - 1, j + 1) + b.d_c * s.LU(i, j) +
                 b.d_d * s.LU(i, j + 1);
        }
        {
            DriveT<R> dr = driving(Hc, Ht, s.BED(i, j), s.BED(i - 1, j), s.PHI(i, j), s.PHI(i - 1, j), dxi, i, ny);
            d -= dr.d_H0 * s.EH(i, j) + dr.d_H1 * s.EH(i - 1, j);
        }
        dv = d;
    }
}

// Staged tile of the JVP: state, e and B in the TMA box layout (rows from
// i0 - 2, columns from j0 - 4), eta and eta-dot of the tile plus a one-cell
// halo.  With 24-entry rows and the 4 x 8 cell patch each warp computes (see
// k_jvp), every stencil access of a warp hits distinct shared-memory banks,
// for 4- and 8-byte values alike.
template <class R>
struct JvpTile {
    static constexpr int T = kTileA, A = 1, NC = T + 2, P = 24, NB = 10;
    Box<R> u, v, eu, ev, H, phi, bed, beta, B, eH;
    R etah[NC][P], detah[NC][P];  // eta H and its derivative along e
};

template <class R>
struct JvpView {
    const JvpTile<R>& t;
    int i0, j0, ny, nx;
    static constexpr int A = 1;
    __device__ int r(int i) const { return i - (i0 - kBoxY); }
    __device__ int c(int j) const { return j - (j0 - kBoxX); }
    __device__ R U(int i, int j) const { return t.u[r(i)][c(j)]; }
    __device__ R V(int i, int j) const { return t.v[r(i)][c(j)]; }
    __device__ R LU(int i, int j) const { return t.eu[r(i)][c(j)]; }
    __device__ R LV(int i, int j) const { return t.ev[r(i)][c(j)]; }
    __device__ R Hc(int i, int j) const { return t.H[r(i)][c(j)]; }
    __device__ R PHI(int i, int j) const { return t.phi[r(i)][c(j)]; }
    __device__ R BED(int i, int j) const { return t.bed[r(i)][c(j)]; }
    __device__ R BETA(int i, int j) const { return t.beta[r(i)][c(j)]; }
    __device__ R BC(int i, int j) const { return t.B[r(i)][c(j)]; }
    __device__ R ETAH(int i, int j) const { return t.etah[i - (i0 - A)][j - (j0 - A)]; }
    __device__ R DETAH(int i, int j) const { return t.detah[i - (i0 - A)][j - (j0 - A)]; }
    __device__ R EH(int i, int j) const { return t.eH[r(i)][c(j)]; }
};

// Viscosity and its derivative along e at one cell, sharing the strain rates
// and one power: eta = B/2 eII^q, eta-dot = eta q eII'/eII (viscosity.cu:63-168).
template <class R, class S>
__device__ __forceinline__ void eta_and_dot(const S& s, R Bc, const PhysR<R>& p, int i, int j, R& eta, R& etad) {
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
    eta = R(0.5) * Bc * glen_pow(eII, p);
    etad = eta * p.gexp * deII / eII;
}

// r_lin = J e - f (- sub) over one level, optional per-block sums of squares.
// Uses VjpArgs with lu/lv/lH carrying e and f_* the right-hand side.  Each
// warp computes a 4 x 8 patch of the 16 x 16 tile.
// The arrays k_jvp stages, in the order of its BoxMaps: u, v, e_u, e_v, H,
// phi, bed, beta, B, e_H.
template <class R, class BLK>
__device__ __forceinline__ void jvp_tile(const VjpArgs<R>& a, int mode, const BoxMaps<JvpTile<R>::NB>& maps,
                                         BLK blk) {
    // mode bit 0: the reference's row conventions; bit 1: mask ignored
    // (the reference's use_mask = False, which reads the mask as 0)
    const bool ref_rows = (mode & 1) != 0, use_mask = (mode & 2) == 0;
    using TT = JvpTile<R>;
    constexpr int NC = TT::NC;
    __shared__ __align__(128) TT T;
    __shared__ double red[3][kTileA * kTileA / 32];
    __shared__ unsigned long long bar;
    const int i0 = blk.y() * kTileA, j0 = blk.x() * kTileA;
    const int ny = a.ny, nx = a.nx;
    {
        Box<R>* const dst[TT::NB] = {&T.u, &T.v, &T.eu, &T.ev, &T.H, &T.phi, &T.bed, &T.beta, &T.B, &T.eH};
        const Arr<R> src[TT::NB] = {a.u, a.v, a.lu, a.lv, a.H, a.phi, a.bed, a.beta, a.B, a.lH};
        if (!stage_boxes<R, TT::NB>(dst, src, maps, i0, j0, &bar, a.err)) return;
    }
    JvpView<R> s{T, i0, j0, ny, nx};
    for (int k = threadIdx.x; k < NC * NC; k += blockDim.x) {
        int r = k / NC, c = k % NC;
        int gi = i0 - 1 + r, gj = j0 - 1 + c;
        R eta, etad;
        eta_and_dot<R>(s, s.BC(gi, gj), a.p, gi, gj, eta, etad);
        const R Hc = s.Hc(gi, gj);
        T.etah[r][c] = eta * Hc;
        T.detah[r][c] = etad * Hc + eta * s.EH(gi, gj);
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int I = i0 + 4 * (w >> 1) + (l >> 3), J = j0 + 8 * (w & 1) + (l & 7);
    double ssu = 0, ssv = 0, ssh = 0;
    const bool f = a.use_forcing != 0;
    auto emit = [&](Arr<R> o, const Arr<R>& fa, const Arr<R>& sa, int i, int j, R val, double& ss) {
        R r = f ? val - fa.at(i, j) : val;
        if (sa.p) r = r - sa.at(i, j);
        o.at(i, j) = r;
        ss += double(r) * double(r);
    };
    if (I < ny && J < nx) {
        const R mk = use_mask ? a.mask.at(I, J) : R(0);
        R dH = mass_jvp<R>(s, a.p, I, J);
        if (ref_rows) dH = (R(1) - mk) * dH;
        else if (mk > R(0.5)) dH = s.EH(I, J);
        emit(a.o_H, a.f_H, a.s_H, I, J, dH, ssh);
        R du = R(0), dv = R(0);
        mom_jvp<R>(s, a.p, I, J, J > 0, I > 0, du, dv);
        // pinned Dirichlet rows; the boundary entries are read only on the boundary
        if (J == 0 && !ref_rows) du = s.LU(I, 0);
        if (I == 0 && !ref_rows) dv = s.LV(0, J);
        emit(a.o_u, a.f_u, a.s_u, I, J, du, ssu);
        if (J == nx - 1) emit(a.o_u, a.f_u, a.s_u, I, nx, ref_rows ? R(0) : s.LU(I, nx), ssu);
        emit(a.o_v, a.f_v, a.s_v, I, J, dv, ssv);
        if (I == ny - 1) emit(a.o_v, a.f_v, a.s_v, ny, J, ref_rows ? R(0) : s.LV(ny, J), ssv);
    }
    if (a.partial) {
        for (int o = 16; o > 0; o >>= 1) {
            ssu += __shfl_down_sync(0xffffffffu, ssu, o);
            ssv += __shfl_down_sync(0xffffffffu, ssv, o);
            ssh += __shfl_down_sync(0xffffffffu, ssh, o);
        }
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
__global__ void __launch_bounds__(kTileA * kTileA)
    k_jvp(VjpArgs<R> a, int mode, const __grid_constant__ BoxMaps<JvpTile<R>::NB> maps) {
    jvp_tile<R>(a, mode, maps, SoloBlock{});
}

}  // namespace glide
