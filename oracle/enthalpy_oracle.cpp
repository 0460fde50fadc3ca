// enthalpy_oracle.cpp -- CPU restatement of the reference's enthalpy column
// solver (test infrastructure; never shipped, never timed as the product).
//
// Follows glide/cuda/enthalpy.cu of JacobDowns/glide:
//   term functions         enthalpy.cu:49-763
//   residual               enthalpy.cu:784-893   (eo_residual)
//   column Newton/Thomas   enthalpy.cu:933-1112  (eo_column_smooth)
//   layer Jacobi           enthalpy.cu:1129-1258 (eo_layer_smooth)
//   omega integration      enthalpy.cu:1277-1372 (eo_compute_omega)
// in binary64, with the reference's layouts: E, E_prev, f_E, omega and the
// outputs (ny, nx, nz) with k fastest; u3d (nz, ny, nx+1); v3d (nz, ny+1, nx).
//
// The reference injects its constants as binary32 literals
// (glide/enthalpy.py:229-246) and folds products of them in binary32; the
// constants below are those binary32 values, and the folded products are
// formed in binary32 the same way, so that this restatement is the binary64
// evaluation of the same discrete operator.
#include <algorithm>
#include <cmath>
#include <vector>

namespace eo {

constexpr float fRHO_I = 910.0f, fRHO_W = 1000.0f, fC_I = 2009.0f, fK_I = 2.1f, fL = 334000.0f;
constexpr float fT_REF = 223.15f, fT_MELT = 273.15f, fBETA = 7.9e-08f, fG = 9.81f, fKTF = 0.1f;
constexpr float fREG = 1.00413490930961e-14f, fREG_YR = 10.0f;

const double RHO_I = fRHO_I, RHO_W = fRHO_W, C_I = fC_I, L_HEAT = fL, T_REF = fT_REF, T_MELT = fT_MELT;
const double K_TEMP_FACTOR = fKTF, MASS_FLUX_REG = fREG, MASS_FLUX_REG_YR = fREG_YR;
const double K_COLD = double(fK_I / fC_I);                 // (K_I/C_I) in binary32
const double E_SCALE = double(fC_I * (fT_MELT - fT_REF));  // (C_I * (T_MELT - T_REF)) in binary32
const double CC_RHO_G = double(fBETA * fRHO_I * fG);       // BETA_CC * RHO_I * GRAVITY in binary32
const double SHARP = double(0.01f);

enum { kHorizAdv = 1, kSigmaDot = 2, kDrainage = 4 };

// enthalpy.cu:49-56
inline double e_pmp(double sigma, double H) {
    double depth = (1.0 - sigma) * H;
    double T_pmp = T_MELT - CC_RHO_G * depth;
    return C_I * (T_pmp - T_REF) / E_SCALE;
}

// enthalpy.cu:60-66
inline double k_diff(double E, double Ep) {
    double z = (E - Ep) * E_SCALE * SHARP;
    z = std::min(std::max(z, -20.0), 20.0);
    double s = 1.0 / (1.0 + std::exp(-z));
    return K_COLD * (1.0 - s + K_TEMP_FACTOR * s);
}

// enthalpy.cu:71-78 (water content) and :85-91 (its derivative)
inline double water(double E, double Ep) {
    double x = (E - Ep) * E_SCALE;
    double ax = SHARP * x;
    ax = std::min(std::max(ax, -20.0), 20.0);
    double sp = (ax > 10.0) ? x : std::log(1.0 + std::exp(ax)) / SHARP;
    return sp / L_HEAT;
}
inline double dwater(double E, double Ep) {
    double z = SHARP * (E - Ep) * E_SCALE;
    z = std::min(std::max(z, -20.0), 20.0);
    double s = 1.0 / (1.0 + std::exp(-z));
    return s / L_HEAT;
}

struct Cfg {
    int ny, nx, nz;
    double dx, dt, drain, h_thin, lf_c;
    int flags;
};

inline size_t cidx(const Cfg& c, int i, int j) { return size_t(i) * c.nx + j; }
inline size_t nidx(const Cfg& c, int i, int j, int k) { return (size_t(i) * c.nx + j) * c.nz + k; }
inline double E_at(const Cfg& c, const double* E, int i, int j, int k) {
    i = std::max(std::min(i, c.ny - 1), 0);
    j = std::max(std::min(j, c.nx - 1), 0);
    k = std::max(std::min(k, c.nz - 1), 0);
    return E[nidx(c, i, j, k)];
}

// Lax-Friedrichs enthalpy flux through one face (enthalpy.cu:573-592)
struct Flux { double res, dl, dr; };
inline Flux face_flux(double q, double El, double Er, double lf_c) {
    double alpha = std::fabs(q) * std::sqrt(1.0 + lf_c);
    return {0.5 * q * (El + Er) - 0.5 * alpha * (Er - El), 0.5 * (q + alpha), 0.5 * (q - alpha)};
}

// Conservative horizontal advection at node (i, j, k) with the centre value
// Ec (enthalpy.cu:667-759)
struct HAdv { double res, diag; };
inline HAdv horiz(const Cfg& c, const double* E, const double* u3d, const double* v3d, const double* H,
                  double Ec, int i, int j, int k) {
    const int ny = c.ny, nx = c.nx, nz = c.nz;
    auto U = [&](int kk, int ii, int jj) {
        kk = std::max(std::min(kk, nz - 1), 0); ii = std::max(std::min(ii, ny - 1), 0);
        jj = std::max(std::min(jj, nx), 0);
        return u3d[(size_t(kk) * ny + ii) * (nx + 1) + jj];
    };
    auto V = [&](int kk, int ii, int jj) {
        kk = std::max(std::min(kk, nz - 1), 0); ii = std::max(std::min(ii, ny), 0);
        jj = std::max(std::min(jj, nx - 1), 0);
        return v3d[(size_t(kk) * (ny + 1) + ii) * nx + jj];
    };
    const double dx_inv = 1.0 / c.dx;
    const double Hc = H[cidx(c, i, j)];
    Flux fl{0, 0, 0}, fr{0, 0, 0}, ft{0, 0, 0}, fb{0, 0, 0};
    const double ul = U(k, i, j), ur = U(k, i, j + 1);
    if (j > 0) {
        double Hm = H[cidx(c, i, j - 1)];
        double q = 0.5 * (Hm + Hc) * ul - 0.5 * std::sqrt(ul * ul + MASS_FLUX_REG) * (Hc - Hm);
        fl = face_flux(q, E_at(c, E, i, j - 1, k), Ec, c.lf_c);
    } else {
        fl = face_flux(0.0, Ec, Ec, c.lf_c);
    }
    if (j < nx - 1) {
        double Hp = H[cidx(c, i, j + 1)];
        double q = 0.5 * (Hc + Hp) * ur - 0.5 * std::sqrt(ur * ur + MASS_FLUX_REG) * (Hp - Hc);
        fr = face_flux(q, Ec, E_at(c, E, i, j + 1, k), c.lf_c);
    } else {
        fr = face_flux(0.0, Ec, Ec, c.lf_c);
    }
    const double vt = V(k, i, j), vb = V(k, i + 1, j);
    if (i > 0) {
        double Hm = H[cidx(c, i - 1, j)];
        double q = 0.5 * (Hm + Hc) * vt - 0.5 * std::sqrt(vt * vt + MASS_FLUX_REG) * (Hm - Hc);
        ft = face_flux(q, Ec, E_at(c, E, i - 1, j, k), c.lf_c);
    } else {
        ft = face_flux(0.0, Ec, Ec, c.lf_c);
    }
    if (i < ny - 1) {
        double Hp = H[cidx(c, i + 1, j)];
        double q = 0.5 * (Hc + Hp) * vb - 0.5 * std::sqrt(vb * vb + MASS_FLUX_REG) * (Hc - Hp);
        fb = face_flux(q, E_at(c, E, i + 1, j, k), Ec, c.lf_c);
    } else {
        fb = face_flux(0.0, Ec, Ec, c.lf_c);
    }
    return {RHO_I * ((fr.res - fl.res) + (ft.res - fb.res)) * dx_inv,
            RHO_I * ((fr.dl - fl.dr) + (ft.dl - fb.dr)) * dx_inv};
}

// One interior or bed row of the column: the E-dependent residual terms other
// than time and horizontal advection, with their tridiagonal coefficients
// (enthalpy.cu:217-509 and :598-640 as assembled by :847-890).
struct Row { double res, a, b, c; };
inline Row vertical_row(const Cfg& c, int k, double Ekm1, double Ek, double Ekp1, const double* om,
                        double h) {
    const double dsig = 1.0 / double(c.nz - 1);
    const double h_inv = 1.0 / h;
    Row row{0, 0, 0, 0};
    if (k == 0) {
        const double Ep0 = e_pmp(0.0, h), Ep1 = e_pmp(dsig, h);
        const double dsh = 0.5 * dsig;
        if (c.flags & kSigmaDot) {
            double wh = 0.5 * (om[0] + om[1]);
            double wp = std::max(wh, 0.0), wn = std::min(wh, 0.0);
            double Fu = wp * Ek + wn * Ekp1, Fb = om[0] * Ek;
            row.res += RHO_I * (Fu - Fb) * (1.0 / dsh);
            row.b += RHO_I * (wp - om[0]) * (1.0 / dsh);
            row.c += RHO_I * wn * (1.0 / dsh);
        }
        double K = k_diff(0.5 * (Ek + Ekp1), 0.5 * (Ep0 + Ep1));
        row.res += (-h_inv * K * (Ekp1 - Ek) / dsig - (0.0 + 0.0)) / dsh;
        double coeff = h_inv * K / (dsig * dsh);
        row.b += coeff;
        row.c += -coeff;
        if (c.flags & kDrainage) {
            row.res += h * RHO_W * L_HEAT * (c.drain * water(Ek, Ep0)) / E_SCALE;
            row.b += h * RHO_W * L_HEAT * c.drain * dwater(Ek, Ep0);
        }
        return row;
    }
    const double Epm = e_pmp(std::max(k - 1, 0) * dsig, h), Epk = e_pmp(k * dsig, h);
    const double Epp = e_pmp(std::min(k + 1, c.nz - 1) * dsig, h);
    if (c.flags & kSigmaDot) {
        double di = 1.0 / dsig;
        double wu = 0.5 * (om[k] + om[std::min(k + 1, c.nz - 1)]);
        double wl = 0.5 * (om[k - 1] + om[k]);
        double up = std::max(wu, 0.0), un = std::min(wu, 0.0);
        double lp = std::max(wl, 0.0), ln = std::min(wl, 0.0);
        double Fu = up * Ek + un * Ekp1, Fl = lp * Ekm1 + ln * Ek;
        row.res += RHO_I * (Fu - Fl) * di;
        row.a += -RHO_I * lp * di;
        row.c += RHO_I * un * di;
        row.b += RHO_I * (up - ln) * di;
    }
    {
        double Ku = k_diff(0.5 * (Ek + Ekp1), 0.5 * (Epk + Epp));
        double Kl = k_diff(0.5 * (Ek + Ekm1), 0.5 * (Epk + Epm));
        double d2 = 1.0 / (dsig * dsig);
        row.res += -h_inv * d2 * (Ku * (Ekp1 - Ek) - Kl * (Ek - Ekm1));
        double dl = h_inv * d2 * Kl, du = h_inv * d2 * Ku;
        row.a += -dl;
        row.c += -du;
        row.b += dl + du;
    }
    if (c.flags & kDrainage) {
        row.res += h * RHO_W * L_HEAT * (c.drain * water(Ek, Epk)) / E_SCALE;
        row.b += h * RHO_W * L_HEAT * c.drain * dwater(Ek, Epk);
    }
    return row;
}

}  // namespace eo

using namespace eo;

extern "C" {

// enthalpy.cu:784-893: out = F(E) - f_E (use_forcing) or F(E)
void eo_residual(double* out, const double* E, const double* E_prev, const double* f_E, const double* u3d,
                 const double* v3d, const double* omega, const double* H, const double* H_prev,
                 const double* E_s, double dx, double dt, double drain, double h_thin, double lf_c, int flags,
                 int use_forcing, int ny, int nx, int nz) {
    Cfg c{ny, nx, nz, dx, dt, drain, h_thin, lf_c, flags};
#pragma omp parallel for schedule(static)
    for (int col = 0; col < ny * nx; ++col) {
        const int i = col / nx, j = col % nx;
        const double h = H[col], hp = H_prev[col];
        double* o = out + size_t(col) * nz;
        if (h < h_thin) {
            for (int k = 0; k < nz; ++k) o[k] = 0.0;
            continue;
        }
        const double* Ec = E + size_t(col) * nz;
        for (int k = 0; k < nz; ++k) {
            if (k == nz - 1) { o[k] = 0.0; continue; }
            double Ek = Ec[k];
            double r = RHO_I * (h * Ek - hp * E_prev[size_t(col) * nz + k]) * (1.0 / dt);
            if (flags & kHorizAdv) r += horiz(c, E, u3d, v3d, H, Ek, i, j, k).res;
            double Ekm1 = k > 0 ? Ec[k - 1] : 0.0;
            Row row = vertical_row(c, k, Ekm1, Ek, Ec[k + 1], omega + size_t(col) * nz, h);
            r += row.res;
            o[k] = use_forcing ? (r - f_E[size_t(col) * nz + k]) : r;
        }
    }
}

// enthalpy.cu:933-1112: delta_E = (column Newton/Thomas result) - E
void eo_column_smooth(double* delta, const double* E, const double* E_prev, const double* f_E,
                      const double* u3d, const double* v3d, const double* omega, const double* H,
                      const double* H_prev, const double* E_s, double dx, double dt, double drain,
                      double h_thin, double lf_c, int flags, int ny, int nx, int nz, int n_newton,
                      double relaxation) {
    Cfg c{ny, nx, nz, dx, dt, drain, h_thin, lf_c, flags};
#pragma omp parallel for schedule(static)
    for (int col = 0; col < ny * nx; ++col) {
        const int i = col / nx, j = col % nx;
        const double h = H[col], hp = H_prev[col];
        const double* Ec = E + size_t(col) * nz;
        double* d = delta + size_t(col) * nz;
        const double dsig = 1.0 / double(nz - 1);
        if (h < h_thin) {
            for (int k = 0; k < nz; ++k) d[k] = std::min(E_s[col], e_pmp(k * dsig, h)) - Ec[k];
            continue;
        }
        std::vector<double> El(Ec, Ec + nz), a(nz), b(nz), cc(nz), rhs(nz), dE(nz);
        for (int it = 0; it < n_newton; ++it) {
            for (int k = 0; k < nz; ++k) {
                if (k == nz - 1) {
                    a[k] = 0.0; b[k] = 1.0; cc[k] = 0.0;
                    rhs[k] = -(El[k] - E_s[col]);
                    continue;
                }
                const size_t ijk = size_t(col) * nz + k;
                double Ek = El[k];
                double r = RHO_I * (h * Ek - hp * E_prev[ijk]) * (1.0 / dt) - f_E[ijk];
                double hdiag = 0.0;
                if (flags & kHorizAdv) {
                    HAdv ha = horiz(c, E, u3d, v3d, H, Ek, i, j, k);
                    r += ha.res;
                    hdiag = ha.diag;
                }
                Row row = vertical_row(c, k, k > 0 ? El[k - 1] : 0.0, Ek, El[k + 1], omega + size_t(col) * nz, h);
                r += row.res;
                a[k] = row.a;
                b[k] = RHO_I * h * (1.0 / dt) + row.b + hdiag;
                cc[k] = row.c;
                rhs[k] = -r;
            }
            for (int k = 1; k < nz; ++k) {
                if (std::fabs(b[k - 1]) < 1e-30) continue;
                double w = a[k] / b[k - 1];
                b[k] -= w * cc[k - 1];
                rhs[k] -= w * rhs[k - 1];
            }
            dE[nz - 1] = rhs[nz - 1] / b[nz - 1];
            for (int k = nz - 2; k >= 0; --k) dE[k] = (rhs[k] - cc[k] * dE[k + 1]) / b[k];
            for (int k = 0; k < nz; ++k) El[k] += relaxation * dE[k];
        }
        for (int k = 0; k < nz; ++k) d[k] = El[k] - Ec[k];
    }
}

// enthalpy.cu:1129-1258: delta_E = -r / diag at every node
void eo_layer_smooth(double* delta, const double* E, const double* E_prev, const double* f_E,
                     const double* u3d, const double* v3d, const double* omega, const double* H,
                     const double* H_prev, const double* E_s, double dx, double dt, double drain,
                     double h_thin, double lf_c, int flags, int ny, int nx, int nz) {
    Cfg c{ny, nx, nz, dx, dt, drain, h_thin, lf_c, flags};
#pragma omp parallel for schedule(static)
    for (int col = 0; col < ny * nx; ++col) {
        const int i = col / nx, j = col % nx;
        const double h = H[col], hp = H_prev[col];
        const double* Ec = E + size_t(col) * nz;
        double* d = delta + size_t(col) * nz;
        for (int k = 0; k < nz; ++k) {
            if (k == nz - 1 || h < h_thin) { d[k] = 0.0; continue; }
            const size_t ijk = size_t(col) * nz + k;
            double Ek = Ec[k];
            double r = RHO_I * (h * Ek - hp * E_prev[ijk]) * (1.0 / dt) - f_E[ijk];
            double diag = RHO_I * h * (1.0 / dt);
            if (flags & kHorizAdv) {
                HAdv ha = horiz(c, E, u3d, v3d, H, Ek, i, j, k);
                r += ha.res;
                diag += ha.diag;
            }
            Row row = vertical_row(c, k, k > 0 ? Ec[k - 1] : 0.0, Ek, Ec[k + 1], omega + size_t(col) * nz, h);
            r += row.res;
            diag += row.b;
            d[k] = (std::fabs(diag) > 1e-30) ? (-r / diag) : 0.0;
        }
    }
}

// enthalpy.cu:1277-1372: omega = H sigma_dot by upward integration
void eo_compute_omega(double* omega, const double* u3d, const double* v3d, const double* H,
                      const double* dh_dt, const double* bmb, double dx, int ny, int nx, int nz) {
#pragma omp parallel for schedule(static)
    for (int col = 0; col < ny * nx; ++col) {
        const int i = col / nx, j = col % nx;
        double* o = omega + size_t(col) * nz;
        const double h = H[col];
        if (h < double(1e-3f)) {
            for (int k = 0; k < nz; ++k) o[k] = 0.0;
            continue;
        }
        auto Hc = [&](int ii, int jj) {
            ii = std::max(std::min(ii, ny - 1), 0); jj = std::max(std::min(jj, nx - 1), 0);
            return H[size_t(ii) * nx + jj];
        };
        const double Hxm = Hc(i, j - 1), Hxp = Hc(i, j + 1), Hym = Hc(i - 1, j), Hyp = Hc(i + 1, j);
        const double dx_inv = 1.0 / dx, dsig = 1.0 / double(nz - 1);
        std::vector<double> div(nz);
        for (int k = 0; k < nz; ++k) {
            const double* uk = u3d + size_t(k) * ny * (nx + 1);
            const double* vk = v3d + size_t(k) * (ny + 1) * nx;
            double ul = uk[size_t(i) * (nx + 1) + j], ur = uk[size_t(i) * (nx + 1) + j + 1];
            double vt = vk[size_t(i) * nx + j], vb = vk[size_t(i + 1) * nx + j];
            double fr = 0, fl = 0, fb = 0, ft = 0;
            if (j < nx - 1) fr = 0.5 * (h + Hxp) * ur - 0.5 * std::sqrt(ur * ur + MASS_FLUX_REG_YR) * (Hxp - h);
            if (j > 0) fl = 0.5 * (Hxm + h) * ul - 0.5 * std::sqrt(ul * ul + MASS_FLUX_REG_YR) * (h - Hxm);
            if (i < ny - 1) fb = 0.5 * (h + Hyp) * vb - 0.5 * std::sqrt(vb * vb + MASS_FLUX_REG_YR) * (h - Hyp);
            if (i > 0) ft = 0.5 * (Hym + h) * vt - 0.5 * std::sqrt(vt * vt + MASS_FLUX_REG_YR) * (Hym - h);
            div[k] = (fr - fl + ft - fb) * dx_inv;
        }
        double w = -bmb[col];
        o[0] = w;
        for (int k = 1; k < nz; ++k) {
            w = w - dsig * (dh_dt[col] + 0.5 * (div[k - 1] + div[k]));
            o[k] = w;
        }
    }
}

double eo_e_scale() { return E_SCALE; }

}  // extern "C"
