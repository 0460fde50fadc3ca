// enthalpy.cu -- handle and C ABI of the enthalpy column solver
// (include/glide_enthalpy.h).  The handle owns the 3-D node arrays (one
// allocation, layer-major) and the 2-D boundary data; the thickness and the
// velocity are read where the caller keeps them (the SSA hierarchy's level-0
// arrays in a coupled run), so a thermal step makes no copies of them.
//
// column_sweep runs all its sweeps without host round trips: each sweep is a
// column-smoother launch writing E + omega delta into a second buffer, a
// layer-smoother launch writing back, a residual launch with per-block
// maxima, and a one-block finisher that applies the reference's stop test
// (glide/enthalpy.py:457-471) on the device and raises a flag; every later
// launch of the sweep sees the flag and returns at once.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "glide_b200.h"
#include "glide_enthalpy.h"
#include "enthalpy_kernels.cuh"

namespace glide {
namespace enth {

static thread_local std::string t_err;

struct Fail {
    int code;
};

[[noreturn]] static void fail(int code, const std::string& msg) {
    t_err = msg;
    throw Fail{code};
}

#define ECU(call)                                                                     \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            fail(GLIDE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

static void check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(GLIDE_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F>
static int guarded(F&& f) {
    try {
        f();
        return GLIDE_OK;
    } catch (const Fail& e) {
        return e.code;
    } catch (const std::exception& e) {
        t_err = e.what();
        return GLIDE_ERR_STATE;
    }
}

// Device-side state of a sweep: initial and last norm, history, stop flag.
struct SweepCtl {
    double r0, last;
    double hist[GLIDE_ENTH_MAX_HISTORY];
    int iters, done;
};

// mode 0: initial norm; mode 1: after a sweep (stop test); mode 2: plain norm
__global__ void __launch_bounds__(1024) k_enth_finish(const double* partial, int nblocks, SweepCtl* ctl, int mode,
                                                       double rtol, double atol) {
    __shared__ double red[32];
    if (mode == 1 && ctl->done) return;
    double m = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) m = fmax(m, partial[b]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int q = 1; q < int(blockDim.x >> 5); ++q) m = fmax(m, red[q]);
    m = fmax(m, red[0]);
    ctl->last = m;
    if (mode == 0) {
        ctl->r0 = m;
        ctl->iters = 0;
        ctl->done = 0;
    } else if (mode == 1) {
        const int it = ctl->iters;
        if (it < GLIDE_ENTH_MAX_HISTORY) ctl->hist[it] = m;
        ctl->iters = it + 1;
        const double rel = ctl->r0 > 0.0 ? m / ctl->r0 : 0.0;
        if (rel < rtol || m < atol) ctl->done = 1;
    }
}

__global__ void k_enth_copy(double* dst, const double* src, size_t n, const int* done) {
    if (done && *(volatile const int*)done) return;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x)
        dst[q] = src[q];
}

__global__ void k_enth_snapshot(double* E_prev, const double* E, size_t n3, double* H_prev, const double* H,
                                int ld_h, int ny, int nx) {
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n3; q += stride) E_prev[q] = E[q];
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < size_t(ny) * nx; q += stride)
        H_prev[q] = H[(q / nx) * ld_h + q % nx];
}

struct Handle {
    int ny, nx, nz;
    double dx;
    size_t plane, n3, nu3, nv3;
    double* arena = nullptr;
    double* f[GLIDE_ENTH_N_FIELDS] = {};
    double* E_alt = nullptr;
    double* rowc = nullptr;  // per-row constants of the on-chip column smoother
    double* dpr = nullptr;   // its Thomas factors d'_k
    double* partial = nullptr;
    SweepCtl* ctl = nullptr;
    SweepCtl* ctl_host = nullptr;
    int nblocks = 0;
    glide_enthalpy_config cfg;
    glide_enthalpy_inputs in;
    int point_blocks = 3;   // resident blocks per SM of the residual / layer kernels (3 to 6)
    // Kernels launched and their algorithmic bytes: the binary64 values each
    // must read and write once.  A residual, column or layer pass moves
    // (5 nz + 7) values per column: E, E_prev, f_E, omega and the output at
    // every level; H, H_prev, E_surface, u, v and two neighbour reads per
    // column.  Sweeps skipped by the device-side stop test move nothing.
    long long launches = 0;
    double alg_bytes = 0;
    void acct(long long n, double bytes) { launches += n; alg_bytes += bytes; }
    double pass_bytes() const { return double(5 * nz + 7) * 8.0 * double(plane); }
    int column_blocks = 4;  // of the column kernel (2 to 6)
    int column_kernel = 1;  // 1 / 2: k_enth_column_s at 6 / 8 blocks per SM; 0: per-thread arrays

    Handle(int ny_, int nx_, int nz_, double dx_) : ny(ny_), nx(nx_), nz(nz_), dx(dx_) {
        plane = size_t(ny) * nx;
        n3 = plane * nz;
        nu3 = size_t(nz) * ny * (nx + 1);
        nv3 = size_t(nz) * (ny + 1) * nx;
        nblocks = int((plane + kColThreads - 1) / kColThreads);
        auto up = [](size_t n) { return (n + 31) / 32 * 32; };  // 256-byte aligned starts
        size_t total = 10 * up(n3) + up(nu3) + up(nv3) + 4 * up(plane) + up(size_t(nblocks)) +
                       up(sizeof(SweepCtl) / sizeof(double) + 1);
        ECU(cudaMalloc(&arena, total * sizeof(double)));
        ECU(cudaMemset(arena, 0, total * sizeof(double)));
        double* p = arena;
        auto take = [&](size_t n) { double* q = p; p += up(n); return q; };
        for (int fld : {GLIDE_ENTH_E, GLIDE_ENTH_E_PREV, GLIDE_ENTH_F_E, GLIDE_ENTH_OMEGA, GLIDE_ENTH_R_E,
                        GLIDE_ENTH_DELTA_E, GLIDE_ENTH_PHI_STRAIN})
            f[fld] = take(n3);
        E_alt = take(n3);
        rowc = take(n3);
        dpr = take(n3);
        f[GLIDE_ENTH_U3D] = take(nu3);
        f[GLIDE_ENTH_V3D] = take(nv3);
        for (int fld : {GLIDE_ENTH_H_PREV, GLIDE_ENTH_E_SURFACE, GLIDE_ENTH_Q_GEO, GLIDE_ENTH_Q_FH})
            f[fld] = take(plane);
        partial = take(size_t(nblocks));
        ctl = reinterpret_cast<SweepCtl*>(take(sizeof(SweepCtl) / sizeof(double) + 1));
        ECU(cudaMallocHost(&ctl_host, sizeof(SweepCtl)));
        // defaults of ColumnSmootherConfig / EnthalpyForcing / EnthalpyTermFlags
        // (glide/enthalpy.py:108-203), as binary64 numbers
        cfg.omega = 1.0;
        cfg.n_newton = 3;
        cfg.relaxation = 1.0;
        cfg.relative_tolerance = 1e-5;
        cfg.absolute_tolerance = 1e-2;
        cfg.lf_c = 1e-12;
        cfg.drain_rate = 0.01 / (365.25 * 86400.0);
        cfg.h_thin = 25.0;
        cfg.term_flags = 7;
        std::memset(&in, 0, sizeof(in));
        in.vel_div = 1.0;
    }
    ~Handle() {
        if (arena) cudaFree(arena);
        if (ctl_host) cudaFreeHost(ctl_host);
    }

    EnthArgs args(double dt, const double* E, bool with_done) const {
        if (!in.H) fail(GLIDE_ERR_STATE, "no thickness bound: call glide_enthalpy_set_inputs first");
        EnthArgs a;
        a.E = E;
        a.E_prev = f[GLIDE_ENTH_E_PREV];
        a.f_E = f[GLIDE_ENTH_F_E];
        a.omega = f[GLIDE_ENTH_OMEGA];
        if (in.u) {
            a.u = in.u; a.ld_u = in.ld_u; a.u_layer = in.u_layer;
        } else {
            a.u = f[GLIDE_ENTH_U3D]; a.ld_u = nx + 1; a.u_layer = (long long)ny * (nx + 1);
        }
        if (in.v) {
            a.v = in.v; a.ld_v = in.ld_v; a.v_layer = in.v_layer;
        } else {
            a.v = f[GLIDE_ENTH_V3D]; a.ld_v = nx; a.v_layer = (long long)(ny + 1) * nx;
        }
        a.H = in.H;
        a.ld_h = in.ld_H;
        a.H_prev = f[GLIDE_ENTH_H_PREV];
        a.E_s = f[GLIDE_ENTH_E_SURFACE];
        a.vel_div = in.vel_div;
        a.dx = dx;
        a.dt = dt;
        a.drain = cfg.drain_rate;
        a.h_thin = cfg.h_thin;
        a.lf_c = cfg.lf_c;
        a.omega_relax = cfg.omega;
        a.relaxation = cfg.relaxation;
        a.flags = cfg.term_flags;
        a.ny = ny;
        a.nx = nx;
        a.nz = nz;
        a.n_newton = cfg.n_newton;
        a.done = with_done ? &ctl->done : nullptr;
        return a;
    }

    dim3 col_grid() const { return dim3(unsigned(nblocks)); }

    void residual(const EnthArgs& a, int use_forcing, cudaStream_t s) {
        if (point_blocks == 3) k_enth_residual<3><<<col_grid(), kColThreads, 0, s>>>(a, f[GLIDE_ENTH_R_E], use_forcing, partial);
        else if (point_blocks == 4) k_enth_residual<4><<<col_grid(), kColThreads, 0, s>>>(a, f[GLIDE_ENTH_R_E], use_forcing, partial);
        else if (point_blocks == 6) k_enth_residual<6><<<col_grid(), kColThreads, 0, s>>>(a, f[GLIDE_ENTH_R_E], use_forcing, partial);
        else k_enth_residual<5><<<col_grid(), kColThreads, 0, s>>>(a, f[GLIDE_ENTH_R_E], use_forcing, partial);
        check_launch("enthalpy residual");
    }
    void column(const EnthArgs& a, double* out, int mode, cudaStream_t s) {
        if (column_kernel >= 1) {
            const size_t smem = size_t(nz) * kColSmemThreads * sizeof(double);
            const unsigned blocks = unsigned((plane + kColSmemThreads - 1) / kColSmemThreads);
            if (column_kernel == 2) k_enth_column_s<8><<<blocks, kColSmemThreads, smem, s>>>(a, out, rowc, dpr, mode);
            else k_enth_column_s<6><<<blocks, kColSmemThreads, smem, s>>>(a, out, rowc, dpr, mode);
            check_launch("enthalpy column smooth (on-chip factors)");
            return;
        }
        if (column_blocks == 2) k_enth_column<2><<<col_grid(), kColThreads, 0, s>>>(a, out, mode);
        else if (column_blocks == 3) k_enth_column<3><<<col_grid(), kColThreads, 0, s>>>(a, out, mode);
        else if (column_blocks == 5) k_enth_column<5><<<col_grid(), kColThreads, 0, s>>>(a, out, mode);
        else if (column_blocks == 6) k_enth_column<6><<<col_grid(), kColThreads, 0, s>>>(a, out, mode);
        else k_enth_column<4><<<col_grid(), kColThreads, 0, s>>>(a, out, mode);
        check_launch("enthalpy column smooth");
    }
    void layer(const EnthArgs& a, double* out, int mode, cudaStream_t s) {
        if (point_blocks == 3) k_enth_layer<3><<<col_grid(), kColThreads, 0, s>>>(a, out, mode);
        else if (point_blocks == 4) k_enth_layer<4><<<col_grid(), kColThreads, 0, s>>>(a, out, mode);
        else if (point_blocks == 6) k_enth_layer<6><<<col_grid(), kColThreads, 0, s>>>(a, out, mode);
        else k_enth_layer<5><<<col_grid(), kColThreads, 0, s>>>(a, out, mode);
        check_launch("enthalpy layer smooth");
    }
    void finish(int mode, cudaStream_t s) {
        k_enth_finish<<<1, 1024, 0, s>>>(partial, nblocks, ctl, mode, cfg.relative_tolerance,
                                         cfg.absolute_tolerance);
        check_launch("enthalpy norm");
    }
    void read_ctl(cudaStream_t s) {
        ECU(cudaMemcpyAsync(ctl_host, ctl, sizeof(SweepCtl), cudaMemcpyDeviceToHost, s));
        ECU(cudaStreamSynchronize(s));
    }
};

}  // namespace enth
}  // namespace glide

using namespace glide::enth;

struct glide_enthalpy {
    Handle* h;
};

static Handle* H(glide_enthalpy_handle h) {
    if (!h || !h->h) fail(GLIDE_ERR_ARG, "null enthalpy handle");
    return h->h;
}
static cudaStream_t S(void* p) { return static_cast<cudaStream_t>(p); }

extern "C" {

const char* glide_enthalpy_last_error(void) { return t_err.c_str(); }

int glide_enthalpy_create(int ny, int nx, int nz, double dx, glide_enthalpy_handle* out) {
    return guarded([&] {
        if (!out) fail(GLIDE_ERR_ARG, "null output pointer");
        if (ny < 1 || nx < 1) fail(GLIDE_ERR_SHAPE, "ny and nx must be positive");
        if (nz < 2 || nz > kMaxNz) fail(GLIDE_ERR_SHAPE, "nz must lie in [2, 64]");
        if (!(dx > 0)) fail(GLIDE_ERR_ARG, "dx must be positive");
        auto* g = new glide_enthalpy{nullptr};
        try {
            g->h = new Handle(ny, nx, nz, dx);
        } catch (...) {
            delete g;
            throw;
        }
        *out = g;
    });
}

int glide_enthalpy_destroy(glide_enthalpy_handle h) {
    return guarded([&] {
        if (!h) return;
        delete h->h;
        delete h;
    });
}

int glide_enthalpy_field_ptr(glide_enthalpy_handle h, int field, void** ptr) {
    return guarded([&] {
        Handle* e = H(h);
        if (field < 0 || field >= GLIDE_ENTH_N_FIELDS) fail(GLIDE_ERR_ARG, "unknown enthalpy field");
        if (!ptr) fail(GLIDE_ERR_ARG, "null output pointer");
        *ptr = e->f[field];
    });
}

int glide_enthalpy_set_config(glide_enthalpy_handle h, const glide_enthalpy_config* c) {
    return guarded([&] {
        Handle* e = H(h);
        if (!c) fail(GLIDE_ERR_ARG, "null config");
        if (c->n_newton < 0) fail(GLIDE_ERR_ARG, "n_newton must be non-negative");
        if (c->term_flags & ~7) fail(GLIDE_ERR_ARG, "unknown term flag");
        e->cfg = *c;
    });
}

int glide_enthalpy_get_config(glide_enthalpy_handle h, glide_enthalpy_config* c) {
    return guarded([&] {
        Handle* e = H(h);
        if (!c) fail(GLIDE_ERR_ARG, "null config");
        *c = e->cfg;
    });
}

int glide_enthalpy_set_tuning(glide_enthalpy_handle h, int key, int value) {
    return guarded([&] {
        Handle* e = H(h);
        if (key == GLIDE_ENTH_TUNE_POINT_BLOCKS) {
            if (value < 3 || value > 6) fail(GLIDE_ERR_ARG, "point blocks per SM must lie in [3, 6]");
            e->point_blocks = value;
        } else if (key == GLIDE_ENTH_TUNE_COLUMN_BLOCKS) {
            if (value < 2 || value > 6) fail(GLIDE_ERR_ARG, "column blocks per SM must lie in [2, 6]");
            e->column_blocks = value;
        } else if (key == GLIDE_ENTH_TUNE_COLUMN_KERNEL) {
            if (value < 0 || value > 2) fail(GLIDE_ERR_ARG, "column kernel must be 0, 1 or 2");
            e->column_kernel = value;
        } else if (key == GLIDE_ENTH_TUNE_COLUMN_L1) {
            const int carve = value ? int(cudaSharedmemCarveoutMaxL1) : int(cudaSharedmemCarveoutDefault);
            ECU(cudaFuncSetAttribute(k_enth_column<2>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
            ECU(cudaFuncSetAttribute(k_enth_column<3>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
            ECU(cudaFuncSetAttribute(k_enth_column<4>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
            ECU(cudaFuncSetAttribute(k_enth_column<5>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
            ECU(cudaFuncSetAttribute(k_enth_column<6>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        } else {
            fail(GLIDE_ERR_ARG, "unknown enthalpy tuning key");
        }
    });
}

int glide_enthalpy_set_inputs(glide_enthalpy_handle h, const glide_enthalpy_inputs* in) {
    return guarded([&] {
        Handle* e = H(h);
        if (!in || !in->H) fail(GLIDE_ERR_ARG, "inputs need a thickness array");
        if (in->ld_H < e->nx) fail(GLIDE_ERR_SHAPE, "ld_H < nx");
        if (in->u && (in->ld_u < e->nx + 1 || in->u_layer < 0)) fail(GLIDE_ERR_SHAPE, "bad u layout");
        if (in->v && (in->ld_v < e->nx || in->v_layer < 0)) fail(GLIDE_ERR_SHAPE, "bad v layout");
        if (!(in->vel_div != 0.0)) fail(GLIDE_ERR_ARG, "vel_div must be non-zero");
        e->in = *in;
    });
}

int glide_enthalpy_snapshot(glide_enthalpy_handle h, void* stream) {
    return guarded([&] {
        Handle* e = H(h);
        if (!e->in.H) fail(GLIDE_ERR_STATE, "no thickness bound");
        k_enth_snapshot<<<1184, 256, 0, S(stream)>>>(e->f[GLIDE_ENTH_E_PREV], e->f[GLIDE_ENTH_E], e->n3,
                                                     e->f[GLIDE_ENTH_H_PREV], e->in.H, e->in.ld_H, e->ny, e->nx);
        check_launch("enthalpy snapshot");
        e->acct(1, 16.0 * (double(e->n3) + double(e->plane)));  // E -> E_prev, H -> H_prev
    });
}

int glide_enthalpy_set_rhs(glide_enthalpy_handle h, void* stream) {
    return guarded([&] {
        Handle* e = H(h);
        EnthArgs a = e->args(1.0, e->f[GLIDE_ENTH_E], false);
        const double e_scale = 2009.0 * (273.15 - 223.15);  // E_SCALE of glide/enthalpy.py
        k_enth_set_rhs<<<e->col_grid(), kColThreads, 0, S(stream)>>>(
            a, e->f[GLIDE_ENTH_F_E], e->f[GLIDE_ENTH_PHI_STRAIN], e->f[GLIDE_ENTH_Q_GEO], e->f[GLIDE_ENTH_Q_FH],
            e_scale);
        check_launch("enthalpy set_rhs");
        e->acct(1, 8.0 * (2.0 * double(e->n3) + 2.0 * double(e->plane)));  // strain heating, Q_geo, Q_fh in; f_E out
    });
}

int glide_enthalpy_residual(glide_enthalpy_handle h, double dt, int use_forcing, double* max_abs, void* stream) {
    return guarded([&] {
        Handle* e = H(h);
        if (!(dt > 0)) fail(GLIDE_ERR_ARG, "dt must be positive");
        EnthArgs a = e->args(dt, e->f[GLIDE_ENTH_E], false);
        e->residual(a, use_forcing, S(stream));
        e->acct(1, e->pass_bytes());
        if (max_abs) {
            e->acct(1, 8.0 * e->nblocks);
            e->finish(2, S(stream));
            e->read_ctl(S(stream));
            *max_abs = e->ctl_host->last;
        }
    });
}

int glide_enthalpy_column_smooth(glide_enthalpy_handle h, double dt, void* stream) {
    return guarded([&] {
        Handle* e = H(h);
        if (!(dt > 0)) fail(GLIDE_ERR_ARG, "dt must be positive");
        EnthArgs a = e->args(dt, e->f[GLIDE_ENTH_E], false);
        e->column(a, e->f[GLIDE_ENTH_DELTA_E], 0, S(stream));
        e->acct(1, e->pass_bytes());
    });
}

int glide_enthalpy_layer_smooth(glide_enthalpy_handle h, double dt, void* stream) {
    return guarded([&] {
        Handle* e = H(h);
        if (!(dt > 0)) fail(GLIDE_ERR_ARG, "dt must be positive");
        EnthArgs a = e->args(dt, e->f[GLIDE_ENTH_E], false);
        e->layer(a, e->f[GLIDE_ENTH_DELTA_E], 0, S(stream));
        e->acct(1, e->pass_bytes());
    });
}

int glide_enthalpy_column_sweep(glide_enthalpy_handle h, double dt, int n_iter, int alternating,
                                glide_enthalpy_stats* stats, void* stream) {
    return guarded([&] {
        Handle* e = H(h);
        if (!(dt > 0)) fail(GLIDE_ERR_ARG, "dt must be positive");
        if (n_iter < 0) fail(GLIDE_ERR_ARG, "negative sweep count");
        cudaStream_t s = S(stream);
        double* E = e->f[GLIDE_ENTH_E];
        EnthArgs home = e->args(dt, E, true);
        EnthArgs alt = e->args(dt, e->E_alt, true);
        // initial norm (its launch must not see a stale stop flag)
        EnthArgs first = home;
        first.done = nullptr;
        e->residual(first, 1, s);
        e->finish(0, s);
        for (int it = 0; it < n_iter; ++it) {
            e->column(home, e->E_alt, 1, s);
            if (alternating) {
                e->layer(alt, E, 1, s);
            } else {
                k_enth_copy<<<1184, 256, 0, s>>>(E, e->E_alt, e->n3, &e->ctl->done);
                check_launch("enthalpy copy");
            }
            e->residual(home, 1, s);
            e->finish(1, s);
        }
        e->read_ctl(s);
        const SweepCtl& c = *e->ctl_host;
        // every launch counts; bytes only for the sweeps that ran (later
        // launches see the stop flag and return at once)
        e->acct(2 + 3LL * n_iter, e->pass_bytes() * (1.0 + 3.0 * c.iters) + 8.0 * e->nblocks * (1.0 + c.iters));
        if (stats) {
            stats->iterations = c.iters;
            stats->initial_norm = c.r0;
            stats->final_norm = c.last;
            for (int q = 0; q < GLIDE_ENTH_MAX_HISTORY; ++q) stats->history[q] = q < c.iters ? c.hist[q] : 0.0;
        }
    });
}

int glide_enthalpy_compute_omega(glide_enthalpy_handle h, const double* dh_dt, int ld_dh, const double* bmb,
                                 int ld_bmb, double dh_div, double omega_div, void* stream) {
    return guarded([&] {
        Handle* e = H(h);
        if (dh_dt && ld_dh < e->nx) fail(GLIDE_ERR_SHAPE, "ld_dh < nx");
        if (bmb && ld_bmb < e->nx) fail(GLIDE_ERR_SHAPE, "ld_bmb < nx");
        if (!dh_dt && !(dh_div != 0.0)) fail(GLIDE_ERR_ARG, "dh_div must be non-zero");
        if (!(omega_div != 0.0)) fail(GLIDE_ERR_ARG, "omega_div must be non-zero");
        EnthArgs a = e->args(1.0, e->f[GLIDE_ENTH_E], false);
        k_enth_omega<<<e->col_grid(), kColThreads, 0, S(stream)>>>(a, e->f[GLIDE_ENTH_OMEGA], dh_dt, ld_dh, bmb,
                                                                  ld_bmb, dh_div, omega_div);
        check_launch("enthalpy omega");
        e->acct(1, 8.0 * (double(e->n3) + 4.0 * double(e->plane)));  // u, v, H, dH/dt in; omega out
    });
}

int glide_enthalpy_frictional_heating(glide_enthalpy_handle h, const double* beta, int ld_beta, double m,
                                      double u_reg, void* stream) {
    return guarded([&] {
        Handle* e = H(h);
        if (!beta || ld_beta < e->nx) fail(GLIDE_ERR_ARG, "bad beta array");
        EnthArgs a = e->args(1.0, e->f[GLIDE_ENTH_E], false);
        k_enth_friction<<<e->col_grid(), kColThreads, 0, S(stream)>>>(a, e->f[GLIDE_ENTH_Q_FH], beta, ld_beta, m,
                                                                     u_reg);
        check_launch("enthalpy frictional heating");
        e->acct(1, 8.0 * 4.0 * double(e->plane));  // beta, u, v in; Q_fh out
    });
}

int glide_enthalpy_arrhenius(glide_enthalpy_handle h, double n_glen, double scale, double* B, int ld_B,
                             void* stream) {
    return guarded([&] {
        Handle* e = H(h);
        if (!B || ld_B < e->nx) fail(GLIDE_ERR_ARG, "bad output array");
        if (!(n_glen > 0) || !(scale != 0.0)) fail(GLIDE_ERR_ARG, "bad n or scale");
        EnthArgs a = e->args(1.0, e->f[GLIDE_ENTH_E], false);
        k_enth_arrhenius<<<e->col_grid(), kColThreads, 0, S(stream)>>>(a, B, ld_B, n_glen, scale);
        check_launch("enthalpy arrhenius");
        e->acct(1, 8.0 * (double(e->n3) + 2.0 * double(e->plane)));  // E, H in; B out
    });
}

int glide_enthalpy_counters(glide_enthalpy_handle h, long long* launches, double* alg_bytes) {
    return guarded([&] {
        Handle* e = H(h);
        if (launches) *launches = e->launches;
        if (alg_bytes) *alg_bytes = e->alg_bytes;
    });
}

}  // extern "C"
