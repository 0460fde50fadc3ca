// tma.cuh -- tensor-memory-accelerator staging of stencil halo tiles.
//
// A stencil block with the 16 x 16 cell tile at (i0, j0) and a one-cell halo
// reads u faces in rows [i0-2, i0+18) and columns [j0-1, j0+18), v faces in
// rows [i0-1, i0+18) and columns [j0-2, j0+18), cells in rows [i0-1, i0+17).
// All of it lies in one box of kBoxH x kBoxW = 20 x 24 elements whose corner
// is (row i0 - 2, column j0 - 4); the column start is a multiple of 4, so the
// copy starts on a 16-byte boundary for 4- and 8-byte elements.  One thread
// issues one cp.async.bulk.tensor per array; all copies complete on one
// mbarrier whose wait is bounded.  The TMA unit fills elements outside the
// array with zeros; tiles on the domain edge then overwrite those with the
// nearest in-array value, the same replicated-edge rule the scalar staging
// applies with clamped indices.
#pragma once

#include <cuda.h>

#include "glide_common.cuh"

namespace glide {

constexpr int kBoxW = 24, kBoxH = 20, kBoxX = 4, kBoxY = 2;

// A box of BH rows and kBoxW columns; BY is its first row's offset above the
// tile (kernels with a two-cell halo stage a taller box).
template <class R, int BH = kBoxH>
using BoxT = R[BH][kBoxW];
template <class R>
using Box = BoxT<R, kBoxH>;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes the initialised barrier visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Polls a staged-tile wait makes before it gives up (each poll itself
// suspends for a bounded, hardware-defined time).
constexpr int kTmaWaitPolls = 1 << 22;

// Waits for the phase with the given parity; gives up after `limit` polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit = kTmaWaitPolls) {
    for (int k = 0; k < limit; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 2-D tiled bulk copy of the box at (column x, row y) of `map` into `dst`.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Bits of a handle's error word set by a staging block.
constexpr int kStageWaitGaveUp = 1;  // the bounded wait for the copies gave up
constexpr int kStageBadMaps = 2;     // the maps did not carry kBoxMapsTag: nothing was copied

constexpr int kBoxMapsTag = 0x474c4d50;

// Tensor maps of the arrays one stencil launch stages (a kernel parameter,
// or an element of a device array the host filled for a grouped launch).
template <int N>
struct BoxMaps {
    CUtensorMap m[N];
    int use;  // 0: stage with clamped scalar loads instead (small levels)
    // polls of the first wait for the copies (kTmaWaitPolls unless a test
    // lowers it to make that wait give up); the wait that lets copies still
    // in flight land after a give-up always uses kTmaWaitPolls
    int wait_polls = kTmaWaitPolls;
    // checked before the first copy: maps read from global memory that do not
    // carry it (not written, or not yet) are never handed to the TMA unit
    int tag = kBoxMapsTag;
};

// Scalar staging of one array into the box layout, indices clamped.
template <class R, int BH = kBoxH, int BY = kBoxY>
__device__ __forceinline__ void stage_box_scalar(BoxT<R, BH>& t, const Arr<R>& a, int i0, int j0) {
    for (int k = threadIdx.x; k < BH * kBoxW; k += blockDim.x) {
        const int r = k / kBoxW, c = k % kBoxW;
        const int gi = clampi(i0 - BY + r, 0, a.rows - 1), gj = clampi(j0 - kBoxX + c, 0, a.cols - 1);
        t[r][c] = ldg(&a.p[size_t(gi) * a.pitch + gj]);
    }
}

// True when the box of the tile at (i0, j0) reaches outside an array of
// rows x cols elements.
template <int BH = kBoxH, int BY = kBoxY>
__device__ __forceinline__ bool box_on_edge(int i0, int j0, int rows, int cols) {
    return i0 - BY < 0 || j0 - kBoxX < 0 || i0 - BY + BH > rows || j0 - kBoxX + kBoxW > cols;
}

// Replace the zero-filled elements outside a rows x cols array by the value
// at the clamped index (which lies inside the box and was copied).
template <class R, int BH = kBoxH, int BY = kBoxY>
__device__ __forceinline__ void box_fixup(BoxT<R, BH>& t, int rows, int cols, int i0, int j0) {
    for (int k = threadIdx.x; k < BH * kBoxW; k += blockDim.x) {
        const int r = k / kBoxW, c = k % kBoxW;
        const int gi = i0 - BY + r, gj = j0 - kBoxX + c;
        if (gi >= 0 && gi < rows && gj >= 0 && gj < cols) continue;
        const int si = clampi(gi, 0, rows - 1) - (i0 - BY), sj = clampi(gj, 0, cols - 1) - (j0 - kBoxX);
        t[r][c] = t[si][sj];
    }
}

// Stage N arrays of one tile.  TMA path: thread 0 issues the copies, every
// thread waits on the barrier, edge tiles are fixed up.  Returns false on
// every thread of the block if the maps fail their check or the wait gave up
// (the error word is then set and the block must return without touching the
// boxes).
template <class R, int N, int BH = kBoxH, int BY = kBoxY>
__device__ __forceinline__ bool stage_boxes(BoxT<R, BH>* const (&dst)[N], const Arr<R> (&src)[N],
                                            const BoxMaps<N>& maps, int i0, int j0, unsigned long long* bar,
                                            int* err) {
    if (maps.use && maps.tag != kBoxMapsTag) {  // the same value on every thread
        if (threadIdx.x == 0) atomicOr(err, kStageBadMaps);
        return false;
    }
    if (!maps.use) {
#pragma unroll
        for (int q = 0; q < N; ++q) stage_box_scalar<R, BH, BY>(*dst[q], src[q], i0, j0);
        __syncthreads();
        return true;
    }
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(bar, unsigned(N * sizeof(BoxT<R, BH>)));
#pragma unroll
        for (int q = 0; q < N; ++q) tma_load_2d(dst[q], &maps.m[q], j0 - kBoxX, i0 - BY, bar);
    }
    const bool ok = __syncthreads_and(mbar_wait(bar, 0, maps.wait_polls));
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(err, kStageWaitGaveUp);
        mbar_wait(bar, 0);  // let copies still in flight land before the block exits
        return false;
    }
    bool edge = false;
#pragma unroll
    for (int q = 0; q < N; ++q) edge |= box_on_edge<BH, BY>(i0, j0, src[q].rows, src[q].cols);
    if (edge) {
#pragma unroll
        for (int q = 0; q < N; ++q)
            if (box_on_edge<BH, BY>(i0, j0, src[q].rows, src[q].cols))
                box_fixup<R, BH, BY>(*dst[q], src[q].rows, src[q].cols, i0, j0);
        __syncthreads();
    }
    return true;
}

// State of a 16 x 16 tile with a one-cell halo in box layout, plus the
// viscosity of the tile cells and their halo (18 x 18, rows padded to 24).
// Box order of the staging maps: u, v, H, phi, bed, beta, B.
template <class R>
struct StateBoxTile {
    static constexpr int NB = 7, NE = 18, P = 24;
    Box<R> u, v, H, phi, bed, beta, B;
    R eta[NE][P];
};

// The accessors of TileView over a StateBoxTile.
template <class R>
struct StateBoxView {
    const StateBoxTile<R>& t;
    int i0, j0, ny, nx;
    __device__ int r(int i) const { return i - (i0 - kBoxY); }
    __device__ int c(int j) const { return j - (j0 - kBoxX); }
    __device__ R U(int i, int j) const { return t.u[r(i)][c(j)]; }
    __device__ R V(int i, int j) const { return t.v[r(i)][c(j)]; }
    __device__ R Hc(int i, int j) const { return t.H[r(i)][c(j)]; }
    __device__ R PHI(int i, int j) const { return t.phi[r(i)][c(j)]; }
    __device__ R BED(int i, int j) const { return t.bed[r(i)][c(j)]; }
    __device__ R BETA(int i, int j) const { return t.beta[r(i)][c(j)]; }
    __device__ R BC(int i, int j) const { return t.B[r(i)][c(j)]; }
    __device__ R ETA(int i, int j) const { return t.eta[i - (i0 - 1)][j - (j0 - 1)]; }
};

template <class R>
__device__ __forceinline__ bool stage_state_boxes(StateBoxTile<R>& t, const BoxMaps<7>& maps, const Arr<R>& u,
                                                  const Arr<R>& v, const Arr<R>& H, const Arr<R>& phi,
                                                  const Arr<R>& bed, const Arr<R>& beta, const Arr<R>& B,
                                                  int i0, int j0, unsigned long long* bar, int* err) {
    Box<R>* const dst[7] = {&t.u, &t.v, &t.H, &t.phi, &t.bed, &t.beta, &t.B};
    const Arr<R> src[7] = {u, v, H, phi, bed, beta, B};
    return stage_boxes<R, 7>(dst, src, maps, i0, j0, bar, err);
}

}  // namespace glide
