// forward_kernels.cuh -- residual, fused Vanka sweep and grounding kernels.
#pragma once

#include "stencil.cuh"
#include "tile.cuh"
#include "tma.cuh"

namespace glide {

constexpr int kTile = 16;

// -------------------------------------------------------------------------
// Residual of the coupled system on one level (residuals.cu:6-333 and the
// host wrapper glide/operators.py:71-127), one thread per cell: the cell's
// mass residual, its left u face and its top v face, plus the right/bottom
// boundary faces for the last column/row.  Optionally subtracts a given
// field (`sub_*`, used to form the coarse FAS right-hand side F(x_c) - R r in
// the same pass) and accumulates per-block sums of squares for the norms.
// -------------------------------------------------------------------------
template <class R>
struct ResidualArgs {
    Arr<R> u, v, H, phi, mask, bed, B, beta, gamma;
    Arr<R> f_u, f_v, f_H;        // forcing, used when use_forcing
    Arr<R> o_u, o_v, o_H;        // outputs
    Arr<R> s_u, s_v, s_H;        // optional subtrahends (p == nullptr: none)
    double* partial;             // optional: 3 sums of squares per block
    int* err;                    // set when a bounded wait gives up
    PhysR<R> p;
    int ny, nx;
    int use_forcing, use_mask;
    int active_set;              // Newton mode (see the mass row below)
};

// The tile's state is staged in box layout (TMA on large levels).  Each warp
// computes a 4 x 8 patch of the 16 x 16 tile; with 24-entry rows the patch's
// stencil reads are bank-conflict free.
// The tile (bx, by) of a grid gx tiles wide; the kernel below runs one tile
// per block, the grouped launches of several hierarchies run the same body.
template <class R, class BLK>
__device__ __forceinline__ void residual_tile(const ResidualArgs<R>& a, const BoxMaps<7>& maps, BLK blk) {
#include "residual_tile.inc"
}

template <class R>
__global__ void __launch_bounds__(256) k_residual(ResidualArgs<R> a,
                                                  const __grid_constant__ BoxMaps<7> maps) {
    const SoloBlock blk{};
#include "residual_tile.inc"
}

// -------------------------------------------------------------------------
// Local 5x5 Vanka systems of every cell for inspection (vanka.cu:801-908,
// operators.py:253-273): the Newton matrix and residual of the cell's five
// unknowns at the current state -- no damping terms -- with the Dirichlet and
// active-set rows pinned as the smoother pins them.  J (ny*nx, 25) row-major,
// r (ny*nx, 5), both contiguous.
// -------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) k_vanka_dump(ResidualArgs<R> a, R* Jout, R* rout) {
    using TileT = Tile<R, kTile, 1, 1>;
    constexpr int NC = TileT::NC;
    __shared__ TileT t;
    const int i0 = blockIdx.y * kTile, j0 = blockIdx.x * kTile;
    const int ny = a.ny, nx = a.nx;
    stage_tile<R, kTile, 1, 1>(t, i0, j0, ny, nx, a.u, a.v, a.H, a.bed, a.beta, &a.phi);
    __syncthreads();
    TileView<R, kTile, 1, 1> s{t, i0, j0, ny, nx};
    for (int k = threadIdx.x; k < NC * NC; k += blockDim.x) {
        int r = k / NC, c = k % NC;
        int gi = i0 - 1 + r, gj = j0 - 1 + c;
        R Bc = ldg(&a.B.p[size_t(clampi(gi, 0, ny - 1)) * a.B.pitch + clampi(gj, 0, nx - 1)]);
        t.eta[r][c] = eta_at<R>(s, Bc, a.p, gi, gj);
    }
    __syncthreads();
    const int i = i0 + threadIdx.x / kTile, j = j0 + threadIdx.x % kTile;
    if (i >= ny || j >= nx) return;
    R x[5] = {s.U(i, j), s.U(i, j + 1), s.V(i, j), s.V(i + 1, j), s.Hc(i, j)};
    R J[25], r[5];
    local_system<R>(s, a.p, i, j, x, J, r);
    r[0] -= a.f_u.at(i, j); r[1] -= a.f_u.at(i, j + 1);
    r[2] -= a.f_v.at(i, j); r[3] -= a.f_v.at(i + 1, j);
    r[4] -= a.f_H.at(i, j);
    if (j == 0) { pin(J, 0); r[0] = x[0]; }
    if (j == nx - 1) { pin(J, 1); r[1] = x[1]; }
    if (i == 0) { pin(J, 2); r[2] = x[2]; }
    if (i == ny - 1) { pin(J, 3); r[3] = x[3]; }
    const R thk = a.gamma.at(i, j);
    if ((x[4] - a.p.dt * r[4]) <= thk) { pin(J, 4); r[4] = x[4] - thk; }
    const size_t c = size_t(i) * nx + j;
#pragma unroll
    for (int q = 0; q < 25; ++q) Jout[c * 25 + q] = J[q];
#pragma unroll
    for (int q = 0; q < 5; ++q) rout[c * 5 + q] = r[q];
}

// Sum the per-block partials in a fixed order and take square roots:
// out[0..2] = |r_u|, |r_v|, |r_H|; out[3] = sqrt of their squares' sum.
// One block of kNormThreads.
constexpr int kNormThreads = 1024;
__device__ __forceinline__ void finish_norms_block(const double* partial, int nblocks, double* out) {
    // thread-strided sums, a fixed shuffle tree per warp, then warp 0 over
    // the 32 warp sums: the same order on every call
    __shared__ double ws[3][32];
    const int t = threadIdx.x, l = t & 31, w = t >> 5;
    double s[3] = {0, 0, 0};
    for (int b = t; b < nblocks; b += kNormThreads)
        for (int q = 0; q < 3; ++q) s[q] += partial[size_t(b) * 3 + q];
    for (int o = 16; o > 0; o >>= 1)
        for (int q = 0; q < 3; ++q) s[q] += __shfl_down_sync(0xffffffffu, s[q], o);
    if (l == 0)
        for (int q = 0; q < 3; ++q) ws[q][w] = s[q];
    __syncthreads();
    if (w == 0) {
        for (int q = 0; q < 3; ++q) s[q] = ws[q][l];
        for (int o = 16; o > 0; o >>= 1)
            for (int q = 0; q < 3; ++q) s[q] += __shfl_down_sync(0xffffffffu, s[q], o);
        if (l == 0) {
            out[0] = sqrt(s[0]);
            out[1] = sqrt(s[1]);
            out[2] = sqrt(s[2]);
            out[3] = sqrt(s[0] + s[1] + s[2]);
        }
    }
}
__global__ void k_finish_norms(const double* partial, int nblocks, double* out);

// -------------------------------------------------------------------------
// Grounded fraction phi = (1-relax) sigmoid(c (bed + 0.917 H)) + relax phi
// (viscosity.cu:17-36).
// -------------------------------------------------------------------------
template <class R>
struct GroundedArgs {
    Arr<R> phi, H, bed;
    R c, relax;
    int ny, nx;
};

template <class R>
__device__ __forceinline__ void grounded_at(const GroundedArgs<R>& a, int i, int j) {
    if (j >= a.nx) return;
    R g = grounded_frac(a.H.at(i, j), a.bed.at(i, j), a.c);
    a.phi.at(i, j) = (R(1) - a.relax) * g + a.relax * a.phi.at(i, j);
}

template <class R>
__global__ void k_grounded(Arr<R> phi, Arr<R> H, Arr<R> bed, R c, R relax, int ny, int nx) {
    const GroundedArgs<R> a{phi, H, bed, c, relax, ny, nx};
    grounded_at(a, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

// -------------------------------------------------------------------------
// One fused additive-Vanka sweep (vanka.cu:478-660 plus the host loop of
// glide/operators.py:194-251): grounding prologue, per-cell damped local
// Newton with the active-set projection, averaging of the face corrections of
// the two cells sharing a face, and the omega-update -- written to a second
// state buffer, because every cell reads its neighbours' old values.
//
// Block = 16x16 own cells + the 16 cells left of the tile + the 16 cells
// above it (288 threads).  The halo cells are solved redundantly so that the
// block owns its faces outright: no atomics, no zero fills, no separate axpy.
// -------------------------------------------------------------------------
enum GammaMode { kGammaArray = 0, kGammaWChi = 1, kGammaWPhi = 2 };

template <class R>
struct SweepArgs {
    Arr<R> u, v, H;              // state in
    Arr<R> uo, vo, Ho;           // state out
    Arr<R> phi, mask, bed, B, beta;
    Arr<R> f_u, f_v, f_H;
    Arr<R> gamma;                // kGammaArray
    Arr<R> wH, chi, chi_c;       // kGammaWChi: wH + chi; kGammaWPhi: wH + (-chi_c[i/2][j/2] + chi)
    int* iters;                  // optional: Newton iterations per cell (pitch = phi.pitch)
    PhysR<R> p;
    R omega, ssa_damping, mc_damping;
    R relax;                     // local Newton step length (the reference fixes 0.5)
    int newton_steps;
    int ny, nx;
    int gmode;                   // GammaMode of grouped launches (the kernel's template fixes it)
};

constexpr int kSweepThreads = kTile * kTile + 2 * kTile;

// MINB = resident blocks per SM the register allocation is fitted to: 1
// keeps every value in registers, 2 doubles the warps that hide the FP64
// dependency latency at the price of some spills; the runtime picks one.
template <class R, bool PHI_LIVE, class BLK>
__device__ __forceinline__ void vanka_sweep_tile(const SweepArgs<R>& a, int gmode, BLK blk) {
    using TileT = Tile<R, kTile, 2, 1>;
    constexpr int NC = TileT::NC;     // 19
    constexpr int ND = kTile + 1;     // deltas for rows/cols [i0-1, i0+16)
    __shared__ TileT t;
    __shared__ R dl[ND][ND][4];
    const int i0 = blk.y() * kTile, j0 = blk.x() * kTile;
    const int ny = a.ny, nx = a.nx;
    stage_tile<R, kTile, 2, 1>(t, i0, j0, ny, nx, a.u, a.v, a.H, a.bed, a.beta, PHI_LIVE ? nullptr : &a.phi);
    __syncthreads();
    TileView<R, kTile, 2, 1> s{t, i0, j0, ny, nx};
    for (int k = threadIdx.x; k < NC * NC; k += blockDim.x) {
        int r = k / NC, c = k % NC;
        int gi = i0 - 2 + r, gj = j0 - 2 + c;
        int ci = clampi(gi, 0, ny - 1), cj = clampi(gj, 0, nx - 1);
        R Bc = ldg(&a.B.p[size_t(ci) * a.B.pitch + cj]);
        t.eta[r][c] = eta_at<R>(s, Bc, a.p, gi, gj);
        if (PHI_LIVE) t.phi[r][c] = grounded_frac(t.H[r][c], t.bed[r][c], a.p.c_ground);
    }
    __syncthreads();

    // which cell does this thread solve?
    int i, j;
    const int tid = threadIdx.x;
    if (tid < kTile * kTile) { i = i0 + tid / kTile; j = j0 + tid % kTile; }
    else if (tid < kTile * kTile + kTile) { i = i0 + (tid - kTile * kTile); j = j0 - 1; }
    else { i = i0 - 1; j = j0 + (tid - kTile * kTile - kTile); }
    const bool live = i >= 0 && i < ny && j >= 0 && j < nx;
    R dH = 0, masked = 0;
    R dd[4] = {0, 0, 0, 0};
    if (live) {
        R x[5] = {s.U(i, j), s.U(i, j + 1), s.V(i, j), s.V(i + 1, j), s.Hc(i, j)};
        R thk;
        if (gmode == kGammaArray) thk = a.gamma.at(i, j);
        else if (gmode == kGammaWChi) thk = a.wH.at(i, j) + a.chi.at(i, j);
        else thk = a.wH.at(i, j) + (-a.chi_c.at(i >> 1, j >> 1) + a.chi.at(i, j));
        masked = tid < kTile * kTile ? a.mask.at(i, j) : R(0);  // halo cells never write it
        R comp[5] = {0, 0, 0, 0, 0};
        R rnorm = 1;
        int k = 0;
        const R tol = R(kNewtonTol);
        while (k < a.newton_steps && rnorm > tol) {
            R J[25], r[5];
            local_system<R>(s, a.p, i, j, x, J, r);
            // forcing is re-read each iteration (L1 hits) to keep registers free
            r[0] -= ldg(&a.f_u.at(i, j)); r[1] -= ldg(&a.f_u.at(i, j + 1));
            r[2] -= ldg(&a.f_v.at(i, j)); r[3] -= ldg(&a.f_v.at(i + 1, j));
            r[4] -= ldg(&a.f_H.at(i, j));
            J[0] -= a.ssa_damping; J[6] -= a.ssa_damping; J[12] -= a.ssa_damping; J[18] -= a.ssa_damping;
            J[24] += a.mc_damping;
            if (j == 0) { pin(J, 0); r[0] = x[0]; }
            if (j == nx - 1) { pin(J, 1); r[1] = x[1]; }
            if (i == 0) { pin(J, 2); r[2] = x[2]; }
            if (i == ny - 1) { pin(J, 3); r[3] = x[3]; }
            if ((x[4] - a.p.dt * r[4]) <= thk) {
                masked = R(1);
                pin(J, 4);
                r[4] = x[4] - thk;
            } else {
                masked = R(0);
            }
            // squared norm of the pre-update local residual (vanka.cu:613)
            rnorm = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3] + r[4] * r[4];
            lu5_solve(J, r, r);
#pragma unroll
            for (int q = 0; q < 5; ++q) {  // compensated (Kahan) update, vanka.cu:617-640
                R y = -a.relax * r[q] - comp[q];
                R tq = x[q] + y;
                comp[q] = (tq - x[q]) - y;
                x[q] = tq;
            }
            x[4] = fmax(x[4], thk);
            ++k;
        }
        if (a.iters && tid < kTile * kTile) a.iters[size_t(i) * a.phi.pitch + j] = k;
        dd[0] = R(0.5) * (x[0] - s.U(i, j));
        dd[1] = R(0.5) * (x[1] - s.U(i, j + 1));
        dd[2] = R(0.5) * (x[2] - s.V(i, j));
        dd[3] = R(0.5) * (x[3] - s.V(i + 1, j));
        dH = x[4] - s.Hc(i, j);
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
        // left face: right half-correction of cell (i, j-1) + left of (i, j)
        R du = (j > 0 ? dl[di][dj - 1][1] : R(0)) + dl[di][dj][0];
        a.uo.at(i, j) = s.U(i, j) + w * du;
        if (j == nx - 1) a.uo.at(i, nx) = s.U(i, nx) + w * dl[di][dj][1];
        R dv = (i > 0 ? dl[di - 1][dj][3] : R(0)) + dl[di][dj][2];
        a.vo.at(i, j) = s.V(i, j) + w * dv;
        if (i == ny - 1) a.vo.at(ny, j) = s.V(ny, j) + w * dl[di][dj][3];
        a.Ho.at(i, j) = s.Hc(i, j) + w * dH;
        a.mask.at(i, j) = masked;
        if (PHI_LIVE) a.phi.at(i, j) = s.PHI(i, j);
    }
}

template <class R, int GMODE, bool PHI_LIVE, int MINB>
__global__ void __launch_bounds__(kSweepThreads, MINB) k_vanka_sweep(SweepArgs<R> a) {
    vanka_sweep_tile<R, PHI_LIVE>(a, GMODE, SoloBlock{});
}

}  // namespace glide
