// transfer_kernels.cuh -- restriction, prolongation and the small pointwise
// kernels of the V-cycle (glide/cuda/transfer.cu semantics; the elementwise
// CuPy expressions of glide/multigrid.py fused into the transfers).
#pragma once

#include "glide_common.cuh"

namespace glide {

enum FieldKind { kFaceU = 0, kFaceV = 1, kCellAvg = 2, kCellMax = 3, kCellMin = 4 };

// Restriction of one field (transfer.cu:2-139) at coarse (J, I).  Coarse
// sizes (nyc, nxc).  Optional second output `copy` receives the same values
// (w_c = x_c).
template <class R>
__device__ __forceinline__ void restrict_at(const Arr<R>& f, const Arr<R>& c, const Arr<R>& copy, int kind,
                                            int nyc, int nxc, int J, int I) {
    R o;
    if (kind == kFaceU) {
        if (J >= nyc || I > nxc) return;
        o = R(0.5) * (f.at(2 * J, 2 * I) + f.at(2 * J + 1, 2 * I));
    } else if (kind == kFaceV) {
        if (J > nyc || I >= nxc) return;
        o = R(0.5) * (f.at(2 * J, 2 * I) + f.at(2 * J, 2 * I + 1));
    } else {
        if (J >= nyc || I >= nxc) return;
        R a = f.at(2 * J, 2 * I), b = f.at(2 * J, 2 * I + 1);
        R cc = f.at(2 * J + 1, 2 * I), d = f.at(2 * J + 1, 2 * I + 1);
        if (kind == kCellAvg) o = R(0.25) * (a + b + cc + d);
        else if (kind == kCellMax) o = fmax(fmax(a, b), fmax(cc, d));
        else o = fmin(fmin(a, b), fmin(cc, d));
    }
    c.at(J, I) = o;
    if (copy.p) copy.at(J, I) = o;
}

template <class R>
__global__ void k_restrict(Arr<R> f, Arr<R> c, Arr<R> copy, int kind, int nyc, int nxc) {
    restrict_at(f, c, copy, kind, nyc, nxc, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

// Several restrictions of one level in one launch: job blockIdx.z.
constexpr int kMaxRestrictJobs = 12;
template <class R>
struct RestrictJobs {
    Arr<R> f[kMaxRestrictJobs], c[kMaxRestrictJobs], copy[kMaxRestrictJobs];
    int kind[kMaxRestrictJobs];
    int nyc, nxc;
};

template <class R>
__global__ void k_restrict_batch(RestrictJobs<R> b) {
    const int q = blockIdx.z;
    restrict_at(b.f[q], b.c[q], b.copy[q], b.kind[q], b.nyc, b.nxc, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

// Bilinear u-face value at fine (j, i) from coarse data addressed through
// `get(J, I)` with coarse sizes (nyc, nxc+1) (transfer.cu:177-229).
template <class R, class G>
__device__ __forceinline__ R bilinear_u(const G& get, int j, int i, int nyc, int nxc) {
    R Jf = (R(j) - R(0.5)) * R(0.5), If = R(i) * R(0.5);
    Jf = fmax(R(0), fmin(Jf, R(nyc - 1)));
    If = fmax(R(0), fmin(If, R(nxc)));
    int Jlo = int(Jf), Ilo = int(If);
    int Jhi = min(Jlo + 1, nyc - 1), Ihi = min(Ilo + 1, nxc);
    R ty = Jf - R(Jlo), tx = If - R(Ilo);
    R v00 = get(Jlo, Ilo), v01 = get(Jlo, Ihi), v10 = get(Jhi, Ilo), v11 = get(Jhi, Ihi);
    return (R(1) - ty) * ((R(1) - tx) * v00 + tx * v01) + ty * ((R(1) - tx) * v10 + tx * v11);
}

// Bilinear v-face value (transfer.cu:270-323).
template <class R, class G>
__device__ __forceinline__ R bilinear_v(const G& get, int j, int i, int nyc, int nxc) {
    R Jf = R(j) * R(0.5), If = (R(i) - R(0.5)) * R(0.5);
    Jf = fmax(R(0), fmin(Jf, R(nyc)));
    If = fmax(R(0), fmin(If, R(nxc - 1)));
    int Jlo = int(Jf), Ilo = int(If);
    int Jhi = min(Jlo + 1, nyc), Ihi = min(Ilo + 1, nxc - 1);
    R ty = Jf - R(Jlo), tx = If - R(Ilo);
    R v00 = get(Jlo, Ilo), v01 = get(Jlo, Ihi), v10 = get(Jhi, Ilo), v11 = get(Jhi, Ihi);
    return (R(1) - ty) * ((R(1) - tx) * v00 + tx * v01) + ty * ((R(1) - tx) * v10 + tx * v11);
}

// Bilinear cell value (transfer.cu:348-395).
template <class R, class G>
__device__ __forceinline__ R bilinear_c(const G& get, int j, int i, int nyc, int nxc) {
    R Jf = (R(j) - R(0.5)) * R(0.5), If = (R(i) - R(0.5)) * R(0.5);
    Jf = fmax(R(0), fmin(Jf, R(nyc - 1)));
    If = fmax(R(0), fmin(If, R(nxc - 1)));
    int Jlo = int(Jf), Ilo = int(If);
    int Jhi = min(Jlo + 1, nyc - 1), Ihi = min(Ilo + 1, nxc - 1);
    R ty = Jf - R(Jlo), tx = If - R(Ilo);
    R v00 = get(Jlo, Ilo), v01 = get(Jlo, Ihi), v10 = get(Jhi, Ilo), v11 = get(Jhi, Ihi);
    return (R(1) - ty) * ((R(1) - tx) * v00 + tx * v01) + ty * ((R(1) - tx) * v10 + tx * v11);
}

// Coarse-grid correction of one field.  With z_c = xc - wc (computed on the
// fly) and P the prolongation of this field:
//   mode 0 (FAS forward, multigrid.py:616-632): x = w + (P z_c + (x - w))
//   mode 1 (adjoint,     multigrid.py:958-967): x = x + P z_c
// `kind`: kFaceU bilinear, kFaceV bilinear, kCellAvg = cell injection,
// kCellMax = cell bilinear; `vquirk` prolongates v data with the u-face
// formula on the v arrays' memory, as the reference does (multigrid.py:212-235).
template <class R>
struct CorrectArgs {
    Arr<R> x, w, xc, wc;
    int kind, mode, vquirk;
    int nyf, nxf;  // fine cell counts
};

template <class R>
__device__ __forceinline__ void correct_at(const CorrectArgs<R>& a, int j, int i) {
    const int nyc = a.nyf / 2, nxc = a.nxf / 2;
    auto zc = [&](int J, int I) { return a.xc.at(J, I) - a.wc.at(J, I); };
    R pz;
    if (a.kind == kFaceU) {
        if (j >= a.nyf || i > a.nxf) return;
        pz = bilinear_u<R>(zc, j, i, nyc, nxc);
    } else if (a.kind == kFaceV) {
        if (j > a.nyf || i >= a.nxf) return;
        if (a.vquirk) {
            // fine flat index in v layout -> (jj, ii) in the u layout the
            // reference's kernel assumes; coarse flat index back to v layout
            const long flat = long(j) * a.nxf + i;
            const int jj = int(flat / (a.nxf + 1)), ii = int(flat % (a.nxf + 1));
            auto zq = [&](int J, int I) {
                const long cf = long(J) * (nxc + 1) + I;
                return zc(int(cf / nxc), int(cf % nxc));
            };
            pz = bilinear_u<R>(zq, jj, ii, nyc, nxc);
        } else {
            pz = bilinear_v<R>(zc, j, i, nyc, nxc);
        }
    } else {
        if (j >= a.nyf || i >= a.nxf) return;
        if (a.kind == kCellAvg) pz = zc(j >> 1, i >> 1);
        else pz = bilinear_c<R>(zc, j, i, nyc, nxc);
    }
    R& x = a.x.at(j, i);
    if (a.mode == 0) {
        R w = a.w.at(j, i);
        x = w + (pz + (x - w));
    } else {
        x = x + pz;
    }
}

// The u, v and H corrections of one level in one launch: job blockIdx.z.
template <class R>
struct CorrectJobs {
    CorrectArgs<R> j[3];
};

template <class R>
__global__ void k_correct_batch(CorrectJobs<R> b) {
    correct_at(b.j[blockIdx.z], blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

// Finest-level snapshot at the top of a V-cycle (multigrid.py:552-556):
// w = x, chi = thklim - H.
template <class R>
struct SnapshotArgs {
    Arr<R> u, v, H, wu, wv, wH, chi;
    R thklim;
    int ny, nx;
};

template <class R>
__device__ __forceinline__ void snapshot_at(const SnapshotArgs<R>& a, int i, int j) {
    if (i < a.ny && j <= a.nx) a.wu.at(i, j) = a.u.at(i, j);
    if (i <= a.ny && j < a.nx) a.wv.at(i, j) = a.v.at(i, j);
    if (i < a.ny && j < a.nx) {
        R h = a.H.at(i, j);
        a.wH.at(i, j) = h;
        if (a.chi.p) a.chi.at(i, j) = a.thklim - h;
    }
}

template <class R>
__global__ void k_snapshot(SnapshotArgs<R> a) {
    snapshot_at(a, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

// f = H_prev / dt + smb (glide/operators.py:275-276)
template <class R>
struct SetRhsArgs {
    Arr<R> fH, Hp, smb;
    R dt;
    int ny, nx;
};

template <class R>
__device__ __forceinline__ void set_rhs_at(const SetRhsArgs<R>& a, int i, int j) {
    if (i < a.ny && j < a.nx) a.fH.at(i, j) = a.Hp.at(i, j) / a.dt + a.smb.at(i, j);
}

template <class R>
__global__ void k_set_rhs(SetRhsArgs<R> a) {
    set_rhs_at(a, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

// Copy of one pitched array (the grouped form of a device-to-device copy).
template <class R>
struct CopyArgs {
    Arr<R> dst, src;
};

template <class R>
__device__ __forceinline__ void copy_at(const CopyArgs<R>& a, int i, int j) {
    if (i < a.src.rows && j < a.src.cols) a.dst.at(i, j) = a.src.at(i, j);
}

// a = s * b + c over a pitched array (c may alias a)
template <class R>
__global__ void k_axpby(Arr<R> a, Arr<R> b, Arr<R> c, R s, int rows, int cols) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (i < rows && j < cols) a.at(i, j) = s * b.at(i, j) + (c.p ? c.at(i, j) : R(0));
}

// d = scale * src, converting the element type
template <class D, class S>
__global__ void k_convert(Arr<D> d, Arr<S> src, double scale, int rows, int cols) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (i < rows && j < cols) {
        D v = D(src.at(i, j));
        d.at(i, j) = scale == 1.0 ? v : D(scale) * v;
    }
}

// d += src (src converted to d's type)
template <class D, class S>
__global__ void k_add_converted(Arr<D> d, Arr<S> src, int rows, int cols) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (i < rows && j < cols) d.at(i, j) = d.at(i, j) + D(src.at(i, j));
}

// Mixed-precision defect correction update of the state: x += y - fl(x) with
// y the low-precision solution started from fl(x); the active set comes from
// the low-precision smoother and masked thicknesses sit exactly on the floor.
template <class D, class S>
__global__ void k_defect_update(Arr<D> u, Arr<D> v, Arr<D> H, Arr<D> mask, Arr<D> gamma, Arr<S> uy,
                                Arr<S> vy, Arr<S> Hy, Arr<S> masky, int ny, int nx) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (i < ny && j <= nx) {
        D x = u.at(i, j);
        u.at(i, j) = x + (D(uy.at(i, j)) - D(S(x)));
    }
    if (i <= ny && j < nx) {
        D x = v.at(i, j);
        v.at(i, j) = x + (D(vy.at(i, j)) - D(S(x)));
    }
    if (i < ny && j < nx) {
        const D m = D(masky.at(i, j));
        D x = H.at(i, j);
        H.at(i, j) = m > D(0.5) ? gamma.at(i, j) : x + (D(Hy.at(i, j)) - D(S(x)));
        mask.at(i, j) = m;
    }
}

// Right-hand side of the Newton correction, -r, in the tangent system's
// precision; active cells take -(H - gamma) so that H + e_H = gamma.
template <class T, class R>
struct TangentRhsArgs {
    Arr<T> fu, fv, fH;
    Arr<R> ru, rv, rH, H, gamma, mask;
    int ny, nx;
};

template <class T, class R>
__device__ __forceinline__ void tangent_rhs_at(const TangentRhsArgs<T, R>& a, int i, int j) {
    if (i < a.ny && j <= a.nx) a.fu.at(i, j) = T(-a.ru.at(i, j));
    if (i <= a.ny && j < a.nx) a.fv.at(i, j) = T(-a.rv.at(i, j));
    if (i < a.ny && j < a.nx)
        a.fH.at(i, j) = T(a.mask.at(i, j) > R(0.5) ? -(a.H.at(i, j) - a.gamma.at(i, j)) : -a.rH.at(i, j));
}

template <class T, class R>
__global__ void k_tangent_rhs(TangentRhsArgs<T, R> a) {
    tangent_rhs_at(a, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

// Newton update x += e (e possibly in lower precision), thickness floored at gamma.
template <class D, class S>
struct NewtonUpdateArgs {
    Arr<D> u, v, H, gamma;
    Arr<S> eu, ev, eH;
    int ny, nx;
};

template <class D, class S>
__device__ __forceinline__ void newton_update_at(const NewtonUpdateArgs<D, S>& a, int i, int j) {
    if (i < a.ny && j <= a.nx) a.u.at(i, j) = a.u.at(i, j) + D(a.eu.at(i, j));
    if (i <= a.ny && j < a.nx) a.v.at(i, j) = a.v.at(i, j) + D(a.ev.at(i, j));
    if (i < a.ny && j < a.nx) a.H.at(i, j) = fmax(a.H.at(i, j) + D(a.eH.at(i, j)), a.gamma.at(i, j));
}

template <class D, class S>
__global__ void k_newton_update(NewtonUpdateArgs<D, S> a) {
    newton_update_at(a, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

template <class R>
struct FillArgs {
    Arr<R> a;
    R val;
};

template <class R>
__device__ __forceinline__ void fill_at(const FillArgs<R>& f, int i, int j) {
    if (i < f.a.rows && j < f.a.cols) f.a.at(i, j) = f.val;
}

template <class R>
__global__ void k_fill(Arr<R> a, R val, int rows, int cols) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (i < rows && j < cols) a.at(i, j) = val;
}

// One stand-alone transfer of one field between caller arrays (the
// Multigrid.restrict_* / prolongate_* helpers, glide/multigrid.py:119-259,
// with the kernels of glide/cuda/transfer.cu).  `op` is a GLIDE_RESTRICT_* /
// GLIDE_PROLONG_* code; (nyf, nxf) are the fine cell counts, the coarse ones
// half of them.  One thread per element of `dst`, whose shape (rows, cols) is
// the launch's.  Codes 12/13 run the u-face formulas over the flat memory of
// v-face arrays, which is what the reference's prolongate_hfacet launches
// (square grids: both layouts then hold (n+1) n elements).
template <class R>
__global__ void k_transfer(Arr<R> src, Arr<R> dst, int op, int nyf, int nxf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (j >= dst.rows || i >= dst.cols) return;
    const int nyc = nyf / 2, nxc = nxf / 2;
    auto c = [&](int J, int I) { return src.at(J, I); };
    R o;
    switch (op) {
        case 0:  // restrict_vfacet (transfer.cu:2-19)
            o = R(0.5) * (src.at(2 * j, 2 * i) + src.at(2 * j + 1, 2 * i));
            break;
        case 1:  // restrict_hfacet (transfer.cu:22-39)
            o = R(0.5) * (src.at(2 * j, 2 * i) + src.at(2 * j, 2 * i + 1));
            break;
        case 2: case 3: case 4: case 5: {  // restrict_cell_{avg,max,min,var} (transfer.cu:42-139)
            const R a = src.at(2 * j, 2 * i), b = src.at(2 * j, 2 * i + 1);
            const R cc = src.at(2 * j + 1, 2 * i), d = src.at(2 * j + 1, 2 * i + 1);
            if (op == 2) o = R(0.25) * (a + b + cc + d);
            else if (op == 3) o = fmax(fmax(a, b), fmax(cc, d));
            else if (op == 4) o = fmin(fmin(a, b), fmin(cc, d));
            else {
                const R mu = R(0.25) * (a + b + cc + d);
                const R d1 = a - mu, d2 = b - mu, d3 = cc - mu, d4 = d - mu;
                o = R(0.25) * (d1 * d1 + d2 * d2 + d3 * d3 + d4 * d4);
            }
            break;
        }
        case 6: {  // prolongate_vfacet_injection (transfer.cu:142-174)
            const int J = j / 2, I = i / 2;
            o = (i % 2 == 0 || I >= nxc) ? c(J, I) : R(0.5) * (c(J, I) + c(J, I + 1));
            break;
        }
        case 7:  // prolongate_vfacet_bilinear (transfer.cu:177-229)
            o = bilinear_u<R>(c, j, i, nyc, nxc);
            break;
        case 8: {  // prolongate_hfacet_injection (transfer.cu:232-267)
            const int J = j / 2, I = i / 2;
            o = (j % 2 == 0 || J >= nyc) ? c(J, I) : R(0.5) * (c(J, I) + c(J + 1, I));
            break;
        }
        case 9:  // prolongate_hfacet_bilinear (transfer.cu:270-323)
            o = bilinear_v<R>(c, j, i, nyc, nxc);
            break;
        case 10:  // prolongate_cell_injection (transfer.cu:326-345)
            o = c(j >> 1, i >> 1);
            break;
        case 11:  // prolongate_cell_bilinear (transfer.cu:348-395)
            o = bilinear_c<R>(c, j, i, nyc, nxc);
            break;
        default: {  // 12, 13: u-face formulas on v-face memory
            const long flat = long(j) * nxf + i;
            const int jj = int(flat / (nxf + 1)), ii = int(flat % (nxf + 1));
            auto q = [&](int J, int I) {
                const long cf = long(J) * (nxc + 1) + I;
                return src.at(int(cf / nxc), int(cf % nxc));
            };
            if (op == 12) {
                const int J = jj / 2, I = ii / 2;
                o = (ii % 2 == 0 || I >= nxc) ? q(J, I) : R(0.5) * (q(J, I) + q(J, I + 1));
            } else {
                o = bilinear_u<R>(q, jj, ii, nyc, nxc);
            }
        }
    }
    dst.at(j, i) = o;
}

}  // namespace glide
