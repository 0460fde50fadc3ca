// glide_common.cuh -- shared definitions of the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace glide {

// rho_i / rho_w as the reference writes it (a binary32 literal, 0.917f); kept
// at its binary32 value in every precision so binary64 results agree with the
// binary64 evaluation of the reference operator.
constexpr double kFlot = double(0.917f);
// Local Newton stopping threshold on the squared local residual (binary32 1e-6).
constexpr double kNewtonTol = double(1e-6f);

// Physical constants of one level (glide/grid.py:28-138 defaults).
struct Phys {
    double n, eps_reg, fr_driving, m, u_reg, water_drag, fr_sliding, calving_rate, fr_calving;
    double thklim;
};

// A pitched 2-D array in device memory: element (r, c) at p[r * pitch + c].
template <class R>
struct Arr {
    R* p = nullptr;
    int rows = 0, cols = 0, pitch = 0;
    __host__ __device__ R& at(int r, int c) const { return p[size_t(r) * pitch + c]; }
};

__host__ __device__ inline int clampi(int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); }

template <class R>
__device__ __forceinline__ R ldg(const R* p) { return __ldg(p); }

// Grid sizes: face arrays u (ny, nx+1) and v (ny+1, nx), cell arrays (ny, nx).
struct Dims {
    int ny, nx;
};

// Block coordinates of a stencil tile.  A kernel launched for one hierarchy
// reads them from the launch (SoloBlock); a grouped launch over several
// hierarchies hands each block the tile it maps to (GroupBlock).
// Both are unsigned, as blockIdx is: the tile origin arithmetic of the
// kernels is unsigned.
struct SoloBlock {
    __device__ __forceinline__ unsigned x() const { return blockIdx.x; }
    __device__ __forceinline__ unsigned y() const { return blockIdx.y; }
    __device__ __forceinline__ unsigned gx() const { return gridDim.x; }
};
struct GroupBlock {
    unsigned bx, by, bz, w;
    __device__ __forceinline__ unsigned x() const { return bx; }
    __device__ __forceinline__ unsigned y() const { return by; }
    __device__ __forceinline__ unsigned gx() const { return w; }
};

}  // namespace glide
