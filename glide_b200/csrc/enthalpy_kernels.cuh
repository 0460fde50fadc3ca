// enthalpy_kernels.cuh -- the conservative enthalpy column solver
// (glide/cuda/enthalpy.cu and glide/enthalpy.py of JacobDowns/glide), binary64.
//
// Layout in HBM: every 3-D node array is layer-major, node (k, i, j) at
// k * plane + i * nx + j (plane = ny * nx).  One thread owns one column
// (i, j) and walks k, so each k step of a warp reads 32 consecutive columns:
// coalesced for every array.  Layer velocities are read with a layer stride;
// stride 0 reads one 2-D field for all layers (the SSA depth-averaged
// velocity, which the reference copies into nz layers).
//
// The reference compiles these kernels with its constants injected as binary32
// literals (glide/enthalpy.py:229-246); products of those literals fold in
// binary32.  The constants below are those binary32 values widened, and the
// folded products are formed in binary32 the same way.
#pragma once

#include <cuda_runtime.h>

namespace glide {
namespace enth {

constexpr int kMaxNz = 64;
constexpr int kColThreads = 128;

constexpr float fRHO_I = 910.0f, fRHO_W = 1000.0f, fC_I = 2009.0f, fK_I = 2.1f, fL_HEAT = 334000.0f;
constexpr float fT_REF = 223.15f, fT_MELT = 273.15f, fBETA_CC = 7.9e-08f, fGRAVITY = 9.81f;
constexpr float fK_TEMP_FACTOR = 0.1f, fMASS_FLUX_REG = 1.00413490930961e-14f, fMASS_FLUX_REG_YR = 10.0f;

constexpr double kRhoI = fRHO_I, kRhoW = fRHO_W, kCI = fC_I, kL = fL_HEAT, kTRef = fT_REF, kTMelt = fT_MELT;
constexpr double kKTF = fK_TEMP_FACTOR, kReg = fMASS_FLUX_REG, kRegYr = fMASS_FLUX_REG_YR;
constexpr double kKCold = double(fK_I / fC_I);                    // (K_I/C_I)
constexpr double kEScale = double(fC_I * (fT_MELT - fT_REF));     // (C_I * (T_MELT - T_REF))
constexpr double kCIoverEScale = kCI / kEScale;                    // folded once, not divided per row
constexpr double kCcRhoG = double(fBETA_CC * fRHO_I * fGRAVITY);  // BETA_CC * RHO_I * GRAVITY
constexpr double kSharp = double(0.01f);                          // K(E) and drainage sharpness

enum { kTermHorizAdv = 1, kTermSigmaDot = 2, kTermDrainage = 4 };

struct EnthArgs {
    const double* E;       // state read (layer-major)
    const double* E_prev;
    const double* f_E;
    const double* omega;
    const double* u;       // layer velocity, u[k * u_layer + i * ld_u + j]
    const double* v;
    const double* H;       // (ny, nx) with leading dimension ld_h
    const double* H_prev;  // (ny, nx) contiguous
    const double* E_s;     // (ny, nx) contiguous
    long long u_layer, v_layer;
    int ld_u, ld_v, ld_h;
    double vel_div;        // velocities are divided by this on read
    double dx, dt, drain, h_thin, lf_c;
    double omega_relax;    // smoother update weight (ColumnSmootherConfig.omega)
    double relaxation;     // Newton step length
    int flags, ny, nx, nz, n_newton;
    const int* done;       // sweep stop flag (nullptr: always run)
};

// ---------------------------------------------------------------- terms
// enthalpy.cu:49-56
__device__ __forceinline__ double e_pmp(double sigma, double H) {
    double depth = (1.0 - sigma) * H;
    double T_pmp = kTMelt - kCcRhoG * depth;
    return (T_pmp - kTRef) * kCIoverEScale;
}

// diffusivity of the switch value s (enthalpy.cu:60-66)
__device__ __forceinline__ double k_of_switch(double s) { return kKCold * (1.0 - s + kKTF * s); }

// Values of the smoothed switches where their argument is clamped at -20 or
// +20 (ice colder or warmer than ~2 K / ~2 kJ kg^-1 from the melting point),
// and the diffusivity there.  They are evaluated once per thread from the
// same expressions, so the clamped branches below return exactly what the
// general path would.
struct Clamped {
    double s_lo, s_hi, sp_lo;
    double k_lo, k_hi;
    __device__ Clamped()
        : s_lo(1.0 / (1.0 + exp(20.0))), s_hi(1.0 / (1.0 + exp(-20.0))),
          sp_lo(log(1.0 + exp(-20.0)) / kSharp), k_lo(k_of_switch(s_lo)), k_hi(k_of_switch(s_hi)) {}
};

// logistic switch 1 / (1 + exp(-z)) with z clamped to [-20, 20]
__device__ __forceinline__ double switch_of(double z, const Clamped& c) {
    if (z <= -20.0) return c.s_lo;
    if (z >= 20.0) return c.s_hi;
    return 1.0 / (1.0 + exp(-z));
}

// enthalpy.cu:60-66
__device__ __forceinline__ double k_diff(double E, double Ep, const Clamped& c) {
    double z = (E - Ep) * kEScale * kSharp;
    if (z <= -20.0) return c.k_lo;
    if (z >= 20.0) return c.k_hi;
    return k_of_switch(1.0 / (1.0 + exp(-z)));
}

// drainage residual and derivative from the softplus sp and switch s
// (enthalpy.cu:71-91, :598-640)
struct Drain { double res, d; };
__device__ __forceinline__ Drain drain_terms(double sp, double s, double drain, double h) {
    return {h * kRhoW * kL * (drain * (sp / kL)) / kEScale, h * kRhoW * kL * drain * (s / kL)};
}

// `cold` is drain_terms at both clamped-low values for this column, which
// is what the general path returns when both arguments are at or below -20.
__device__ __forceinline__ Drain drainage(double Ek, double Ep, double drain, double h, const Clamped& c,
                                          const Drain& cold) {
    double x = (Ek - Ep) * kEScale;
    double ax = kSharp * x;
    double z = kSharp * (Ek - Ep) * kEScale;
    if (ax <= -20.0 && z <= -20.0) return cold;
    double sp;
    if (ax <= -20.0) sp = c.sp_lo;
    else if (ax > 10.0) sp = x;
    else sp = log(1.0 + exp(ax)) / kSharp;
    double s = switch_of(z, c);
    return drain_terms(sp, s, drain, h);
}

// Lax-Friedrichs enthalpy flux through a face with mass flux q; sq = sqrt(1 + lf_c)
// (enthalpy.cu:573-592)
struct Flux { double res, dl, dr; };
__device__ __forceinline__ Flux face_flux(double q, double El, double Er, double sq) {
    double alpha = fabs(q) * sq;
    return {0.5 * q * (El + Er) - 0.5 * alpha * (Er - El), 0.5 * (q + alpha), 0.5 * (q - alpha)};
}

// Per-column horizontal context: thicknesses of the column and its four
// neighbours and which faces are interior.
struct ColumnCtx {
    int i, j;
    size_t c;              // column offset i * nx + j
    double h, h_prev, h_inv;
    double Hxm, Hxp, Hym, Hyp;
};

__device__ __forceinline__ ColumnCtx column_ctx(const EnthArgs& a, int i, int j) {
    ColumnCtx x;
    x.i = i; x.j = j;
    x.c = size_t(i) * a.nx + j;
    const double* H = a.H;
    x.h = H[size_t(i) * a.ld_h + j];
    x.h_prev = a.H_prev[x.c];
    x.h_inv = 1.0 / x.h;
    x.Hxm = j > 0 ? H[size_t(i) * a.ld_h + j - 1] : 0.0;
    x.Hxp = j < a.nx - 1 ? H[size_t(i) * a.ld_h + j + 1] : 0.0;
    x.Hym = i > 0 ? H[size_t(i - 1) * a.ld_h + j] : 0.0;
    x.Hyp = i < a.ny - 1 ? H[size_t(i + 1) * a.ld_h + j] : 0.0;
    return x;
}

// Mass fluxes H u through the four faces of a column at layer k, with the
// Lax-Friedrichs thickness flux of the momentum solver (enthalpy.cu:690-745);
// boundary faces carry none.  With a layer-independent velocity they are
// the same for every k and are evaluated once per column.
struct FaceQ { double l, r, t, b; };
__device__ __forceinline__ FaceQ face_q(const EnthArgs& a, const ColumnCtx& x, int k) {
    const double* uk = a.u + k * a.u_layer + size_t(x.i) * a.ld_u;
    const double* vk = a.v + k * a.v_layer;
    FaceQ q{0.0, 0.0, 0.0, 0.0};
    if (x.j > 0) {
        double ul = uk[x.j] / a.vel_div;
        q.l = 0.5 * (x.Hxm + x.h) * ul - 0.5 * sqrt(ul * ul + kReg) * (x.h - x.Hxm);
    }
    if (x.j < a.nx - 1) {
        double ur = uk[x.j + 1] / a.vel_div;
        q.r = 0.5 * (x.h + x.Hxp) * ur - 0.5 * sqrt(ur * ur + kReg) * (x.Hxp - x.h);
    }
    if (x.i > 0) {
        double vt = vk[size_t(x.i) * a.ld_v + x.j] / a.vel_div;
        q.t = 0.5 * (x.Hym + x.h) * vt - 0.5 * sqrt(vt * vt + kReg) * (x.Hym - x.h);
    }
    if (x.i < a.ny - 1) {
        double vb = vk[size_t(x.i + 1) * a.ld_v + x.j] / a.vel_div;
        q.b = 0.5 * (x.h + x.Hyp) * vb - 0.5 * sqrt(vb * vb + kReg) * (x.h - x.Hyp);
    }
    return q;
}

struct HAdv { double res, diag; };

// The four horizontal neighbours of node (k, i, j) in the state array; a
// neighbour across the domain edge reads as 0 and is not used.
struct Nbr { double l, r, t, b; };
__device__ __forceinline__ Nbr neighbours(const EnthArgs& a, const ColumnCtx& x, int k) {
    const double* Ek = a.E + size_t(k) * (size_t(a.ny) * a.nx);
    Nbr n{0.0, 0.0, 0.0, 0.0};
    if (x.j > 0) n.l = Ek[x.c - 1];
    if (x.j < a.nx - 1) n.r = Ek[x.c + 1];
    if (x.i > 0) n.t = Ek[x.c - a.nx];
    if (x.i < a.ny - 1) n.b = Ek[x.c + a.nx];
    return n;
}

// Conservative horizontal advection at (i, j, k) with centre value Ec and
// the neighbours n read from the state array (enthalpy.cu:667-759).  sq =
// sqrt(1 + lf_c), dx_inv = 1 / dx.
__device__ __forceinline__ HAdv horiz_vals(const EnthArgs& a, const ColumnCtx& x, double Ec, const Nbr& n,
                                           const FaceQ& q, double sq, double dx_inv) {
    Flux fl = x.j > 0 ? face_flux(q.l, n.l, Ec, sq) : face_flux(0.0, Ec, Ec, sq);
    Flux fr = x.j < a.nx - 1 ? face_flux(q.r, Ec, n.r, sq) : face_flux(0.0, Ec, Ec, sq);
    Flux ft = x.i > 0 ? face_flux(q.t, Ec, n.t, sq) : face_flux(0.0, Ec, Ec, sq);
    Flux fb = x.i < a.ny - 1 ? face_flux(q.b, n.b, Ec, sq) : face_flux(0.0, Ec, Ec, sq);
    return {kRhoI * ((fr.res - fl.res) + (ft.res - fb.res)) * dx_inv,
            kRhoI * ((fr.dl - fl.dr) + (ft.dl - fb.dr)) * dx_inv};
}

// Per-column horizontal-advection context: the hoisted face fluxes (valid
// for every k when the velocity is layer-independent) and the constants.
struct HCtx {
    FaceQ q;
    bool flat;  // velocity independent of the layer
    double sq, dx_inv;
    __device__ HCtx(const EnthArgs& a, const ColumnCtx& x) {
        flat = a.u_layer == 0 && a.v_layer == 0;
        sq = sqrt(1.0 + a.lf_c);
        dx_inv = 1.0 / a.dx;
        q = flat ? face_q(a, x, 0) : FaceQ{0.0, 0.0, 0.0, 0.0};
    }
};

// Vertical terms of row k < nz - 1: sigma advection, diffusion, drainage with
// their tridiagonal coefficients (enthalpy.cu:217-509).  K_lo / K_up are the
// diffusivities of the interfaces below and above node k, which the caller
// carries from row to row (the reference evaluates each twice, from the same
// arguments).
struct Vert { double adv, dif, drn; double a, b_dif, b_adv, b_drn, c; };

// Per-column constants of the vertical terms: 1 / dsig, 1 / dsig^2 and the
// drainage of ice below both switches' clamp (the same expressions the
// per-row code evaluated).
struct ColTerms {
    double di, d2;
    Drain cold;
    __device__ ColTerms(const EnthArgs& a, const Clamped& c, double h, double dsig)
        : di(1.0 / dsig), d2(1.0 / (dsig * dsig)), cold(drain_terms(c.sp_lo, c.s_lo, a.drain, h)) {}
};

__device__ __forceinline__ Vert vertical(const EnthArgs& a, int k, double Ekm1, double Ek, double Ekp1,
                                         double Epk, double K_lo, double K_up, double om_m, double om_k,
                                         double om_p, double h, double h_inv, double dsig, const Clamped& cl,
                                         const ColTerms& ct) {
    Vert r{0, 0, 0, 0, 0, 0, 0, 0};
    if (k == 0) {
        const double dsh = 0.5 * dsig, dsh_inv = 1.0 / dsh;
        if (a.flags & kTermSigmaDot) {
            double wh = 0.5 * (om_k + om_p);
            double wp = fmax(wh, 0.0), wn = fmin(wh, 0.0);
            double Fu = wp * Ek + wn * Ekp1, Fb = om_k * Ek;
            r.adv = kRhoI * (Fu - Fb) * dsh_inv;
            r.b_adv = kRhoI * (wp - om_k) * dsh_inv;
            r.c = kRhoI * wn * dsh_inv;
        }
        r.dif = (-h_inv * K_up * (Ekp1 - Ek) / dsig - 0.0) / dsh;
        double coeff = h_inv * K_up / (dsig * dsh);
        r.b_dif = coeff;
        r.c += -coeff;
    } else {
        const double di = ct.di;
        if (a.flags & kTermSigmaDot) {
            double wu = 0.5 * (om_k + om_p), wl = 0.5 * (om_m + om_k);
            double up = fmax(wu, 0.0), un = fmin(wu, 0.0), lp = fmax(wl, 0.0), ln = fmin(wl, 0.0);
            double Fu = up * Ek + un * Ekp1, Fl = lp * Ekm1 + ln * Ek;
            r.adv = kRhoI * (Fu - Fl) * di;
            r.a = -kRhoI * lp * di;
            r.c = kRhoI * un * di;
            r.b_adv = kRhoI * (up - ln) * di;
        }
        const double d2 = ct.d2;
        r.dif = -h_inv * d2 * (K_up * (Ekp1 - Ek) - K_lo * (Ek - Ekm1));
        double dl = h_inv * d2 * K_lo, du = h_inv * d2 * K_up;
        r.a += -dl;
        r.c += -du;
        r.b_dif = dl + du;
    }
    if (a.flags & kTermDrainage) {
        Drain d = drainage(Ek, Epk, a.drain, h, cl, ct.cold);
        r.drn = d.res;
        r.b_drn = d.d;
    }
    return r;
}

__device__ __forceinline__ bool stopped(const int* done) { return done && *(volatile const int*)done; }

// Inputs of row k of a column that do not depend on the column iterate:
// E_prev, f_E (when used), omega of node k + 1 and the frozen horizontal
// neighbours.  The kernels below load row k + 1's while row k is computed,
// so the walk up the column does not wait on memory at every row.  E_prev,
// f_E and omega are each read by one thread only, so they are loaded with
// the streaming hint (evict first): in L2 they then give way to the column
// kernel's per-thread Newton/Thomas arrays and to the neighbour rows of E,
// which other blocks read again.
struct RowIn { double ep, fe, om_p; Nbr nb; };
__device__ __forceinline__ RowIn row_inputs(const EnthArgs& a, const ColumnCtx& x, int k, bool hadv,
                                            bool forcing) {
    const size_t plane = size_t(a.ny) * a.nx;
    const size_t n = size_t(k) * plane + x.c;
    RowIn r{__ldcs(a.E_prev + n), forcing ? __ldcs(a.f_E + n) : 0.0, __ldcs(a.omega + n + plane),
            Nbr{0.0, 0.0, 0.0, 0.0}};
    if (hadv) r.nb = neighbours(a, x, k);
    return r;
}
__device__ __forceinline__ RowIn no_row() { return RowIn{0.0, 0.0, 0.0, Nbr{0.0, 0.0, 0.0, 0.0}}; }

// Horizontal advection of row k from its loaded neighbours.
__device__ __forceinline__ HAdv row_horiz(const EnthArgs& a, const ColumnCtx& x, const HCtx& hc, int k, double Ec,
                                          const Nbr& nb) {
    return horiz_vals(a, x, Ec, nb, hc.flat ? hc.q : face_q(a, x, k), hc.sq, hc.dx_inv);
}

// ------------------------------------------------------------- residual
// enthalpy.cu:784-893.  out (layer-major) = F(E) - f_E, or F(E) without
// forcing; partial[block] = max |out| over the block's nodes.
template <int MINB>
__global__ void __launch_bounds__(kColThreads, MINB) k_enth_residual(EnthArgs a, double* out, int use_forcing,
                                                                  double* partial) {
    __shared__ double red[kColThreads / 32];
    if (stopped(a.done)) return;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int nz = a.nz;
    const size_t plane = size_t(a.ny) * a.nx;
    double mx = 0.0;
    if (col < a.ny * a.nx) {
        const int i = col / a.nx, j = col % a.nx;
        const ColumnCtx x = column_ctx(a, i, j);
        if (x.h < a.h_thin) {
            for (int k = 0; k < nz; ++k) out[k * plane + x.c] = 0.0;
        } else {
            const Clamped cl;
            const HCtx hc(a, x);
            const double dsig = 1.0 / double(nz - 1), inv_dt = 1.0 / a.dt;
            const ColTerms ct(a, cl, x.h, dsig);
            const double* E = a.E + x.c;
            const double* om = a.omega + x.c;
            double Ekm1 = 0.0, Ek = E[0], Ekp1 = E[plane];
            double Epk = e_pmp(0.0, x.h), Epp = e_pmp(dsig, x.h);
            double K_lo = 0.0;
            double om_m = 0.0, om_k = om[0];
            const bool hadv = (a.flags & kTermHorizAdv) != 0;
            RowIn in = row_inputs(a, x, 0, hadv, use_forcing);
            for (int k = 0; k < nz - 1; ++k) {
                const RowIn in_n = k + 1 < nz - 1 ? row_inputs(a, x, k + 1, hadv, use_forcing) : no_row();
                const double E_n = (k + 2 < nz) ? E[size_t(k + 2) * plane] : 0.0;
                const double om_p = in.om_p;
                const double K_up = k_diff(0.5 * (Ek + Ekp1), 0.5 * (Epk + Epp), cl);
                double r = kRhoI * (x.h * Ek - x.h_prev * in.ep) * inv_dt;
                if (hadv) r += row_horiz(a, x, hc, k, Ek, in.nb).res;
                Vert vt = vertical(a, k, Ekm1, Ek, Ekp1, Epk, K_lo, K_up, om_m, om_k, om_p, x.h, x.h_inv, dsig, cl, ct);
                r += vt.adv;
                r += vt.dif;
                r += vt.drn;
                if (use_forcing) r = r - in.fe;
                out[k * plane + x.c] = r;
                mx = fmax(mx, fabs(r));
                // slide the window
                Ekm1 = Ek; Ek = Ekp1; Ekp1 = E_n;
                Epk = Epp;
                Epp = e_pmp(double(k + 2 < nz ? k + 2 : nz - 1) * dsig, x.h);
                K_lo = K_up;
                om_m = om_k; om_k = om_p;
                in = in_n;
            }
            out[size_t(nz - 1) * plane + x.c] = 0.0;
        }
    }
    if (partial) {
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = red[0];
            for (int q = 1; q < kColThreads / 32; ++q) m = fmax(m, red[q]);
            partial[blockIdx.x] = m;
        }
    }
}

// --------------------------------------------------------- column smoother
// enthalpy.cu:933-1112: per column, n_newton damped Newton steps on the
// column with the horizontal neighbours frozen, each a tridiagonal (Thomas)
// solve.  mode 0 writes delta_E = E_col - E; mode 1 writes the updated state
// E + omega_relax (E_col - E).  Rows are assembled and eliminated in one
// upward pass (Thomas in its c', d' form), then back-substituted.
template <int MINB>
__global__ void __launch_bounds__(kColThreads, MINB) k_enth_column(EnthArgs a, double* out, int mode) {
    if (stopped(a.done)) return;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.ny * a.nx) return;
    const int nz = a.nz;
    const size_t plane = size_t(a.ny) * a.nx;
    const int i = col / a.nx, j = col % a.nx;
    const ColumnCtx x = column_ctx(a, i, j);
    const double* E = a.E + x.c;
    const double dsig = 1.0 / double(nz - 1);
    const double Es = a.E_s[x.c];
    double El[kMaxNz], cp[kMaxNz], dp[kMaxNz];
    if (x.h < a.h_thin) {
        // thin ice: driven to min(E_surface, E_pmp) (enthalpy.cu:963-973)
        for (int k = 0; k < nz; ++k) {
            double Ek = E[size_t(k) * plane];
            double d = fmin(Es, e_pmp(k * dsig, x.h)) - Ek;
            out[size_t(k) * plane + x.c] = mode ? Ek + a.omega_relax * d : d;
        }
        return;
    }
    for (int k = 0; k < nz; ++k) El[k] = E[size_t(k) * plane];
    const Clamped cl;
    const HCtx hc(a, x);
    const ColTerms ct(a, cl, x.h, dsig);
    const double inv_dt = 1.0 / a.dt;
    const double* om = a.omega + x.c;
    const double bt = kRhoI * x.h * inv_dt;  // time-term diagonal
    const bool hadv = (a.flags & kTermHorizAdv) != 0;
    for (int it = 0; it < a.n_newton; ++it) {
        double Epk = e_pmp(0.0, x.h), Epp = e_pmp(dsig, x.h);
        double K_lo = 0.0, om_m = 0.0, om_k = om[0];
        double c_prev = 0.0, d_prev = 0.0;
        // the iterate window of row k and the inputs of row k + 1 are
        // loaded before row k is assembled
        double Ekm1 = 0.0, Ek = El[0], Ekp1 = El[1];
        RowIn in = row_inputs(a, x, 0, hadv, true);
        for (int k = 0; k < nz - 1; ++k) {
            const RowIn in_n = k + 1 < nz - 1 ? row_inputs(a, x, k + 1, hadv, true) : no_row();
            const double E_n = k + 2 < nz ? El[k + 2] : 0.0;
            const double om_p = in.om_p;
            const double K_up = k_diff(0.5 * (Ek + Ekp1), 0.5 * (Epk + Epp), cl);
            double r = kRhoI * (x.h * Ek - x.h_prev * in.ep) * inv_dt - in.fe;
            double hd = 0.0;
            if (hadv) {
                HAdv ha = row_horiz(a, x, hc, k, Ek, in.nb);
                r += ha.res;
                hd = ha.diag;
            }
            Vert vt = vertical(a, k, Ekm1, Ek, Ekp1, Epk, K_lo, K_up, om_m, om_k, om_p, x.h, x.h_inv, dsig, cl, ct);
            r += vt.adv;
            r += vt.dif;
            r += vt.drn;
            const double b = bt + vt.b_dif + vt.b_adv + vt.b_drn + hd;
            // elimination: b' = b - a c'_{k-1}; c'_k = c / b'; d'_k = (rhs - a d'_{k-1}) / b'
            const double bp = b - vt.a * c_prev;
            const double inv = 1.0 / bp;
            c_prev = vt.c * inv;
            d_prev = (-r - vt.a * d_prev) * inv;
            cp[k] = c_prev;
            dp[k] = d_prev;
            Epk = Epp;
            Epp = e_pmp(double(k + 2 < nz ? k + 2 : nz - 1) * dsig, x.h);
            K_lo = K_up;
            om_m = om_k; om_k = om_p;
            Ekm1 = Ek; Ek = Ekp1; Ekp1 = E_n;
            in = in_n;
        }
        // surface Dirichlet row: E = E_surface (a = c = 0, b = 1)
        double xk = -(El[nz - 1] - Es);
        El[nz - 1] += a.relaxation * xk;
#pragma unroll 4
        for (int k = nz - 2; k >= 0; --k) {
            xk = dp[k] - cp[k] * xk;
            El[k] += a.relaxation * xk;
        }
    }
    for (int k = 0; k < nz; ++k) {
        const double Ek = E[size_t(k) * plane];
        const double d = El[k] - Ek;
        out[size_t(k) * plane + x.c] = mode ? Ek + a.omega_relax * d : d;
    }
}

// ---------------------------------------- column smoother, on-chip factors
// The same smoother as k_enth_column, organised so that nothing per column
// has to live in local memory:
//  * the Thomas factor c'_k sits in shared memory, laid out [k][thread] so a
//    warp's accesses fall in distinct banks; d'_k goes to a layer-major
//    scratch array (`dpr`) and the Newton iterate lives in `out`, both
//    coalesced, with an in-flight footprint (2 nz values per resident
//    column) that stays in L2;
//  * on the first Newton iteration the part of each row that does not depend
//    on the column iterate -- the old time level, the forcing and, for a
//    layer-independent velocity, the frozen neighbours' share of the
//    horizontal flux -- is folded into one constant per row, stored in
//    `rowc`; later iterations read it and omega instead of the seven row
//    inputs, and the horizontal diagonal is a column constant;
//  * the back substitution loads d'_k and the iterate four rows ahead, so its
//    serial chain does not wait on memory at every row.
// The rows are the same expressions regrouped (the time term split as
// rho H E / dt - rho H_prev E_prev / dt, the horizontal flux as its diagonal
// times E plus the neighbours' share), so results agree with k_enth_column
// to rounding.  The last Newton iteration's back substitution writes the
// smoother output directly.  Dynamic shared memory: nz blockDim doubles.
constexpr int kColSmemThreads = 64;

// Per-column constants of k_enth_column_s.
struct ColS {
    double bt, ct_old, hd_flat, Es;
    bool hadv, fold;
};

// One Newton step of one column: rows assembled and eliminated upward,
// then back-substituted.  FIRST: the iterate is E, the row inputs are read
// and the row constants written; otherwise the iterate is `El` and the row
// constants are read.
template <bool FIRST>
__device__ __forceinline__ void column_newton_step(const EnthArgs& a, const ColumnCtx& x, const Clamped& cl,
                                                   const HCtx& hc, const ColTerms& ct, const ColS& cs,
                                                   const double* E, double* El, double* C, double* Dp,
                                                   double* cps, int bd, bool last, int mode) {
    const int nz = a.nz;
    const size_t plane = size_t(a.ny) * a.nx;
    const double dsig = 1.0 / double(nz - 1);
    const double* om = a.omega + x.c;
    const double* src = FIRST ? E : El;
    double Epk = e_pmp(0.0, x.h), Epp = e_pmp(dsig, x.h);
    double K_lo = 0.0, om_m = 0.0, om_k = om[0];
    double c_prev = 0.0, d_prev = 0.0;
    double Ekm1 = 0.0, Ek = src[0], Ekp1 = src[plane];
    // row k + 1's inputs are loaded while row k is assembled
    RowIn in = FIRST ? row_inputs(a, x, 0, cs.hadv, true) : no_row();
    double Cn = FIRST ? 0.0 : C[0];
    double om_n = FIRST ? 0.0 : om[plane];
    for (int k = 0; k < nz - 1; ++k) {
        const double E_n = k + 2 < nz ? src[size_t(k + 2) * plane] : 0.0;
        double ck, om_p;
        RowIn in_n = no_row();
        if (FIRST) {
            if (k + 1 < nz - 1) in_n = row_inputs(a, x, k + 1, cs.hadv, true);
            // the row constant: old time level, forcing, frozen neighbours
            ck = -cs.ct_old * in.ep - in.fe;
            if (cs.fold) ck += row_horiz(a, x, hc, k, 0.0, in.nb).res;
            C[size_t(k) * plane] = ck;
            om_p = in.om_p;
        } else {
            ck = Cn;
            om_p = om_n;
            if (k + 1 < nz - 1) {
                Cn = C[size_t(k + 1) * plane];
                om_n = om[size_t(k + 2) * plane];
            }
        }
        const double K_up = k_diff(0.5 * (Ek + Ekp1), 0.5 * (Epk + Epp), cl);
        double r = cs.bt * Ek + ck;
        double hd = cs.hd_flat;
        if (cs.fold) {
            r += cs.hd_flat * Ek;
        } else if (cs.hadv) {
            const Nbr nb = FIRST ? in.nb : neighbours(a, x, k);
            HAdv ha = row_horiz(a, x, hc, k, Ek, nb);
            r += ha.res;
            hd = ha.diag;
        }
        Vert vt = vertical(a, k, Ekm1, Ek, Ekp1, Epk, K_lo, K_up, om_m, om_k, om_p, x.h, x.h_inv, dsig, cl, ct);
        r += vt.adv;
        r += vt.dif;
        r += vt.drn;
        const double b = cs.bt + vt.b_dif + vt.b_adv + vt.b_drn + hd;
        // elimination: b' = b - a c'_{k-1}; c'_k = c / b'; d'_k = (rhs - a d'_{k-1}) / b'
        const double bp = b - vt.a * c_prev;
        const double inv = 1.0 / bp;
        c_prev = vt.c * inv;
        d_prev = (-r - vt.a * d_prev) * inv;
        cps[size_t(k) * bd] = c_prev;
        Dp[size_t(k) * plane] = d_prev;
        Epk = Epp;
        Epp = e_pmp(double(k + 2 < nz ? k + 2 : nz - 1) * dsig, x.h);
        K_lo = K_up;
        om_m = om_k; om_k = om_p;
        Ekm1 = Ek; Ek = Ekp1; Ekp1 = E_n;
        if (FIRST) in = in_n;
    }
    // surface Dirichlet row: E = E_surface (a = c = 0, b = 1), then back
    // substitution; the last Newton step writes the smoother output.  The
    // iterate, d'_k and (on the last step) the input state of row k are
    // loaded kPre rows ahead into a register ring.
    const double top = src[size_t(nz - 1) * plane];
    double xk = -(top - cs.Es);
    double en = top + a.relaxation * xk;
    if (last) {
        const double E0 = E[size_t(nz - 1) * plane];
        El[size_t(nz - 1) * plane] = mode ? E0 + a.omega_relax * (en - E0) : en - E0;
    } else {
        El[size_t(nz - 1) * plane] = en;
    }
    constexpr int kPre = 4;
    const bool want_e = last && !FIRST;
    double ps[kPre], pd[kPre], pe[kPre];
#pragma unroll
    for (int q = 0; q < kPre; ++q) {
        const int k = nz - 2 - q;
        ps[q] = k >= 0 ? src[size_t(k) * plane] : 0.0;
        pd[q] = k >= 0 ? Dp[size_t(k) * plane] : 0.0;
        pe[q] = (want_e && k >= 0) ? E[size_t(k) * plane] : 0.0;
    }
#pragma unroll kPre
    for (int q = 0; q < nz - 1; ++q) {
        const int k = nz - 2 - q, slot = q % kPre;
        const double sk = ps[slot], dk = pd[slot], ek = pe[slot];
        const int kn = k - kPre;
        if (kn >= 0) {
            ps[slot] = src[size_t(kn) * plane];
            pd[slot] = Dp[size_t(kn) * plane];
            if (want_e) pe[slot] = E[size_t(kn) * plane];
        }
        xk = dk - cps[size_t(k) * bd] * xk;
        en = sk + a.relaxation * xk;
        if (last) {
            const double E0 = FIRST ? sk : ek;
            El[size_t(k) * plane] = mode ? E0 + a.omega_relax * (en - E0) : en - E0;
        } else {
            El[size_t(k) * plane] = en;
        }
    }
}

template <int MINB>
__global__ void __launch_bounds__(kColSmemThreads, MINB)
    k_enth_column_s(EnthArgs a, double* out, double* rowc, double* dpr, int mode) {
    extern __shared__ double sm[];
    if (stopped(a.done)) return;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.ny * a.nx) return;
    const int nz = a.nz;
    const size_t plane = size_t(a.ny) * a.nx;
    const int i = col / a.nx, j = col % a.nx;
    const ColumnCtx x = column_ctx(a, i, j);
    const double* E = a.E + x.c;
    double* El = out + x.c;
    const double dsig = 1.0 / double(nz - 1);
    const double Es = a.E_s[x.c];
    if (x.h < a.h_thin) {
        // thin ice: driven to min(E_surface, E_pmp) (enthalpy.cu:963-973)
        for (int k = 0; k < nz; ++k) {
            double Ek = E[size_t(k) * plane];
            double d = fmin(Es, e_pmp(k * dsig, x.h)) - Ek;
            El[size_t(k) * plane] = mode ? Ek + a.omega_relax * d : d;
        }
        return;
    }
    if (a.n_newton <= 0) {
        for (int k = 0; k < nz; ++k) El[size_t(k) * plane] = mode ? E[size_t(k) * plane] : 0.0;
        return;
    }
    double* cps = sm + threadIdx.x;  // c'_k at cps[k * blockDim.x]
    const Clamped cl;
    const HCtx hc(a, x);
    const ColTerms ct(a, cl, x.h, dsig);
    ColS cs;
    const double inv_dt = 1.0 / a.dt;
    cs.bt = kRhoI * x.h * inv_dt;          // time-term diagonal
    cs.ct_old = kRhoI * x.h_prev * inv_dt;  // time-term weight of E_prev
    cs.hadv = (a.flags & kTermHorizAdv) != 0;
    cs.fold = cs.hadv && hc.flat;           // horizontal flux folded into the row constants
    cs.hd_flat = cs.fold ? horiz_vals(a, x, 0.0, Nbr{0.0, 0.0, 0.0, 0.0}, hc.q, hc.sq, hc.dx_inv).diag : 0.0;
    cs.Es = Es;
    double* C = rowc + x.c;
    double* Dp = dpr + x.c;
    column_newton_step<true>(a, x, cl, hc, ct, cs, E, El, C, Dp, cps, blockDim.x, a.n_newton == 1, mode);
    for (int it = 1; it < a.n_newton; ++it)
        column_newton_step<false>(a, x, cl, hc, ct, cs, E, El, C, Dp, cps, blockDim.x, it + 1 == a.n_newton, mode);
}

// ---------------------------------------------------------- layer smoother
// enthalpy.cu:1129-1258: pointwise Jacobi, delta = -r / J_kk.  One thread per
// column walking k.  mode 0 writes delta_E, mode 1 the updated state.
template <int MINB>
__global__ void __launch_bounds__(kColThreads, MINB) k_enth_layer(EnthArgs a, double* out, int mode) {
    if (stopped(a.done)) return;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.ny * a.nx) return;
    const int nz = a.nz;
    const size_t plane = size_t(a.ny) * a.nx;
    const int i = col / a.nx, j = col % a.nx;
    const ColumnCtx x = column_ctx(a, i, j);
    const double* E = a.E + x.c;
    if (x.h < a.h_thin) {
        for (int k = 0; k < nz; ++k) out[size_t(k) * plane + x.c] = mode ? E[size_t(k) * plane] : 0.0;
        return;
    }
    const Clamped cl;
    const HCtx hc(a, x);
    const double dsig = 1.0 / double(nz - 1), inv_dt = 1.0 / a.dt;
    const ColTerms ct(a, cl, x.h, dsig);
    const double* om = a.omega + x.c;
    double Ekm1 = 0.0, Ek = E[0], Ekp1 = E[plane];
    double Epk = e_pmp(0.0, x.h), Epp = e_pmp(dsig, x.h);
    double K_lo = 0.0, om_m = 0.0, om_k = om[0];
    const bool hadv = (a.flags & kTermHorizAdv) != 0;
    RowIn in = row_inputs(a, x, 0, hadv, true);
    for (int k = 0; k < nz - 1; ++k) {
        const RowIn in_n = k + 1 < nz - 1 ? row_inputs(a, x, k + 1, hadv, true) : no_row();
        const double E_n = (k + 2 < nz) ? E[size_t(k + 2) * plane] : 0.0;
        const double om_p = in.om_p;
        const double K_up = k_diff(0.5 * (Ek + Ekp1), 0.5 * (Epk + Epp), cl);
        const size_t n = size_t(k) * plane + x.c;
        double r = kRhoI * (x.h * Ek - x.h_prev * in.ep) * inv_dt - in.fe;
        double diag = kRhoI * x.h * inv_dt;
        if (hadv) {
            HAdv ha = row_horiz(a, x, hc, k, Ek, in.nb);
            r += ha.res;
            diag += ha.diag;
        }
        Vert vt = vertical(a, k, Ekm1, Ek, Ekp1, Epk, K_lo, K_up, om_m, om_k, om_p, x.h, x.h_inv, dsig, cl, ct);
        r += vt.adv;
        r += vt.dif;
        r += vt.drn;
        diag += vt.b_dif + vt.b_adv + vt.b_drn;
        const double d = (fabs(diag) > 1e-30) ? (-r / diag) : 0.0;
        out[n] = mode ? Ek + a.omega_relax * d : d;
        Ekm1 = Ek; Ek = Ekp1; Ekp1 = E_n;
        Epk = Epp;
        Epp = e_pmp(double(k + 2 < nz ? k + 2 : nz - 1) * dsig, x.h);
        K_lo = K_up;
        om_m = om_k; om_k = om_p;
        in = in_n;
    }
    const size_t top = size_t(nz - 1) * plane + x.c;
    out[top] = mode ? E[size_t(nz - 1) * plane] : 0.0;
}

// ------------------------------------------------------------ omega
// enthalpy.cu:1277-1372: omega = H sigma_dot integrated upward from
// omega(0) = -bmb.  dh_dt: explicit array, or (H - H_prev) / dh_div when
// dh_dt is null (glide/model.py:237-258).  Velocities are read undivided
// (the reference evaluates this in m/a); omega is divided by omega_div.
__global__ void __launch_bounds__(kColThreads) k_enth_omega(EnthArgs a, double* omega, const double* dh_dt,
                                                               int ld_dh, const double* bmb, int ld_bmb,
                                                               double dh_div, double omega_div) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.ny * a.nx) return;
    const int nz = a.nz;
    const size_t plane = size_t(a.ny) * a.nx;
    const int i = col / a.nx, j = col % a.nx;
    const double* H = a.H;
    const double h = H[size_t(i) * a.ld_h + j];
    const size_t c = size_t(i) * a.nx + j;
    if (h < double(1e-3f)) {
        for (int k = 0; k < nz; ++k) omega[size_t(k) * plane + c] = 0.0;
        return;
    }
    auto Hc = [&](int ii, int jj) {
        ii = ii < 0 ? 0 : (ii > a.ny - 1 ? a.ny - 1 : ii);
        jj = jj < 0 ? 0 : (jj > a.nx - 1 ? a.nx - 1 : jj);
        return H[size_t(ii) * a.ld_h + jj];
    };
    const double Hxm = Hc(i, j - 1), Hxp = Hc(i, j + 1), Hym = Hc(i - 1, j), Hyp = Hc(i + 1, j);
    const double dx_inv = 1.0 / a.dx, dsig = 1.0 / double(nz - 1);
    const double dh = dh_dt ? dh_dt[size_t(i) * ld_dh + j] : (h - a.H_prev[c]) / dh_div;
    double w = bmb ? -bmb[size_t(i) * ld_bmb + j] : -0.0;
    omega[c] = w / omega_div;
    // horizontal divergence of the thickness flux at level k
    auto div_at = [&](int k) {
        const double* uk = a.u + k * a.u_layer + size_t(i) * a.ld_u;
        const double* vk = a.v + k * a.v_layer;
        const double ul = uk[j], ur = uk[j + 1];
        const double vt = vk[size_t(i) * a.ld_v + j], vb = vk[size_t(i + 1) * a.ld_v + j];
        double fr = 0.0, fl = 0.0, fb = 0.0, ft = 0.0;
        if (j < a.nx - 1) fr = 0.5 * (h + Hxp) * ur - 0.5 * sqrt(ur * ur + kRegYr) * (Hxp - h);
        if (j > 0) fl = 0.5 * (Hxm + h) * ul - 0.5 * sqrt(ul * ul + kRegYr) * (h - Hxm);
        if (i < a.ny - 1) fb = 0.5 * (h + Hyp) * vb - 0.5 * sqrt(vb * vb + kRegYr) * (h - Hyp);
        if (i > 0) ft = 0.5 * (Hym + h) * vt - 0.5 * sqrt(vt * vt + kRegYr) * (Hym - h);
        return (fr - fl + ft - fb) * dx_inv;
    };
    // a depth-independent velocity (layer stride 0) gives every level the
    // same divergence: evaluate it once
    const bool flat = a.u_layer == 0 && a.v_layer == 0;
    const double div_flat = flat ? div_at(0) : 0.0;
    double div_prev = 0.0;
    for (int k = 0; k < nz; ++k) {
        const double div = flat ? div_flat : div_at(k);
        if (k > 0) {
            w = w - dsig * (dh + 0.5 * (div_prev + div));
            omega[size_t(k) * plane + c] = w / omega_div;
        }
        div_prev = div;
    }
}

// ------------------------------------------------------------- forcing
// EnthalpyOperators.set_rhs (glide/enthalpy.py:473-519): f_E = H phi_strain /
// E_SCALE below the surface, plus (Q_geo + Q_fh) / (dsig/2 E_SCALE) at the bed,
// 0 at the surface.  e_scale is the host-side E_SCALE of glide/enthalpy.py.
__global__ void __launch_bounds__(kColThreads) k_enth_set_rhs(EnthArgs a, double* f_E, const double* phi_strain,
                                                                 const double* Q_geo, const double* Q_fh,
                                                                 double e_scale) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.ny * a.nx) return;
    const int nz = a.nz;
    const size_t plane = size_t(a.ny) * a.nx;
    const int i = col / a.nx, j = col % a.nx;
    const size_t c = size_t(i) * a.nx + j;
    const double h = a.H[size_t(i) * a.ld_h + j];
    const double dsig_half = 0.5 * (1.0 / double(nz - 1));
    // distinct arrays: the unrolled loop issues several levels' loads ahead
    // of their stores
    const double* __restrict__ ps = phi_strain + c;
    double* __restrict__ fe = f_E + c;
#pragma unroll 4
    for (int k = 0; k < nz - 1; ++k) {
        double f = h * ps[size_t(k) * plane] / e_scale;
        if (k == 0) f += (Q_geo[c] + Q_fh[c]) / (dsig_half * e_scale);
        fe[size_t(k) * plane] = f;
    }
    fe[size_t(nz - 1) * plane] = 0.0;
}

// Q_fh = beta |u_b|^(m+1) from the bed-layer velocity (glide/model.py:224-235)
__global__ void k_enth_friction(EnthArgs a, double* Q_fh, const double* beta, int ld_beta, double m,
                                double u_reg) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.ny * a.nx) return;
    const int i = col / a.nx, j = col % a.nx;
    const double* u0 = a.u + size_t(i) * a.ld_u;
    const double uc = 0.5 * (u0[j + 1] / a.vel_div + u0[j] / a.vel_div);
    const double vc = 0.5 * (a.v[size_t(i + 1) * a.ld_v + j] / a.vel_div + a.v[size_t(i) * a.ld_v + j] / a.vel_div);
    const double speed = sqrt(uc * uc + vc * vc + u_reg * u_reg);
    Q_fh[size_t(i) * a.nx + j] = beta[size_t(i) * ld_beta + j] * pow(speed, m + 1.0);
}

// Depth-averaged rate factor B = mean_k(A)^(-1/n) / scale (Paterson-Budd with
// water-content enhancement, glide/enthalpy.py:600-643).  Host-side constants
// of glide/enthalpy.py (binary64), sigma as numpy.linspace gives it.
__global__ void __launch_bounds__(kColThreads, 8) k_enth_arrhenius(EnthArgs a, double* B, int ld_B, double n_glen,
                                                                   double scale) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.ny * a.nx) return;
    const int nz = a.nz;
    const size_t plane = size_t(a.ny) * a.nx;
    const int i = col / a.nx, j = col % a.nx;
    const size_t c = size_t(i) * a.nx + j;
    const double h = a.H[size_t(i) * a.ld_h + j];
    const double step = 1.0 / double(nz - 1);
    const double E_SCALE = 2009.0 * (273.15 - 223.15), cc = 7.9e-8 * 910.0 * 9.81;
    auto rate = [&](int k) {
        const double sig = (k == nz - 1) ? 1.0 : k * step;
        const double depth = (1.0 - sig) * h;
        const double T_pmp = 273.15 - cc * depth;
        const double Ek = a.E[size_t(k) * plane + c];
        const double T = fmin(Ek * E_SCALE / 2009.0 + 223.15, T_pmp);
        const bool cold = T < 263.15;
        const double Af = cold ? 3.985e-13 : 1.916e3, Qf = cold ? 60e3 : 139e3;
        double A = Af * exp(-Qf / (8.314 * fmax(T, 1.0)));
        const double w = fmax(Ek * E_SCALE - 2009.0 * (T_pmp - 223.15), 0.0) / 334000.0;
        return A * (1.0 + 181.25 * w);
    };
    // numpy's pairwise sum of a short contiguous axis: below 8 terms in order;
    // else 8 interleaved partial sums combined pairwise, then the rest in order
    double sum = 0.0;
    if (nz < 8) {
        for (int k = 0; k < nz; ++k) sum += rate(k);
    } else {
        double r[8];
        for (int q = 0; q < 8; ++q) r[q] = rate(q);
        const int n8 = nz - nz % 8;
        for (int k = 8; k < n8; k += 8)
            for (int q = 0; q < 8; ++q) r[q] += rate(k + q);
        sum = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (int k = n8; k < nz; ++k) sum += rate(k);
    }
    const double A_avg = sum / double(nz);
    B[size_t(i) * ld_B + j] = pow(A_avg, -1.0 / n_glen) / scale;
}

}  // namespace enth
}  // namespace glide
