// tile.cuh -- shared-memory halo tiles for the stencil kernels.
//
// A block owns a T x T tile of cells with origin (i0, j0).  The staged cell
// region is rows/cols [i0-A, i0+T+B); u faces are staged for rows
// [i0-A-1, i0+T+B+1) and columns [j0-A, j0+T+B+1); v faces for rows
// [i0-A, i0+T+B+1) and columns [j0-A-1, j0+T+B+1).  Every staged element is
// read from global memory with its indices clamped into the array, which is
// exactly the reference's boundary rule (replicated edge values), so the
// stencil code indexes the tile without any clamping.
#pragma once

#include "glide_common.cuh"

namespace glide {

// P > 0 pads every row to P entries (P = 8 mod 16 makes a 4 x 8 cell patch
// per warp bank-conflict free for 4- and 8-byte values).
template <class R, int T, int A, int B, int P = 0>
struct Tile {
    static constexpr int NC = T + A + B;
    static constexpr int WU = P ? P : NC + 1, WV = P ? P : NC + 2, WC = P ? P : NC;
    R u[NC + 2][WU];
    R v[NC + 1][WV];
    R H[NC][WC];
    R phi[NC][WC];
    R bed[NC][WC];
    R beta[NC][WC];
    R eta[NC][WC];
};

template <class R, int T, int A, int B, int P = 0>
struct TileView {
    const Tile<R, T, A, B, P>& t;
    int i0, j0, ny, nx;
    __device__ R U(int i, int j) const { return t.u[i - (i0 - A - 1)][j - (j0 - A)]; }
    __device__ R V(int i, int j) const { return t.v[i - (i0 - A)][j - (j0 - A - 1)]; }
    __device__ R Hc(int i, int j) const { return t.H[i - (i0 - A)][j - (j0 - A)]; }
    __device__ R PHI(int i, int j) const { return t.phi[i - (i0 - A)][j - (j0 - A)]; }
    __device__ R BED(int i, int j) const { return t.bed[i - (i0 - A)][j - (j0 - A)]; }
    __device__ R BETA(int i, int j) const { return t.beta[i - (i0 - A)][j - (j0 - A)]; }
    __device__ R ETA(int i, int j) const { return t.eta[i - (i0 - A)][j - (j0 - A)]; }
};

// Stage u, v, H, bed, beta (and phi when `phi` is non-null) for the tile.
template <class R, int T, int A, int B, int P = 0>
__device__ void stage_tile(Tile<R, T, A, B, P>& t, int i0, int j0, int ny, int nx, const Arr<R>& u,
                           const Arr<R>& v, const Arr<R>& H, const Arr<R>& bed, const Arr<R>& beta,
                           const Arr<R>* phi) {
    constexpr int NC = Tile<R, T, A, B, P>::NC;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int k = tid; k < (NC + 2) * (NC + 1); k += nt) {
        int r = k / (NC + 1), c = k % (NC + 1);
        int gi = clampi(i0 - A - 1 + r, 0, ny - 1), gj = clampi(j0 - A + c, 0, nx);
        t.u[r][c] = ldg(&u.p[size_t(gi) * u.pitch + gj]);
    }
    for (int k = tid; k < (NC + 1) * (NC + 2); k += nt) {
        int r = k / (NC + 2), c = k % (NC + 2);
        int gi = clampi(i0 - A + r, 0, ny), gj = clampi(j0 - A - 1 + c, 0, nx - 1);
        t.v[r][c] = ldg(&v.p[size_t(gi) * v.pitch + gj]);
    }
    for (int k = tid; k < NC * NC; k += nt) {
        int r = k / NC, c = k % NC;
        int gi = clampi(i0 - A + r, 0, ny - 1), gj = clampi(j0 - A + c, 0, nx - 1);
        size_t o = size_t(gi) * H.pitch + gj;  // all cell arrays share one pitch
        t.H[r][c] = ldg(&H.p[o]);
        t.bed[r][c] = ldg(&bed.p[o]);
        t.beta[r][c] = ldg(&beta.p[o]);
        if (phi) t.phi[r][c] = ldg(&phi->p[o]);
    }
}

}  // namespace glide
