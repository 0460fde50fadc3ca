// noalloc.cu -- residual and residual norms without any device allocation.
//
// Who needs this: host programs that own every byte of device memory through
// their own allocator or a fixed budget set at start-up -- an Earth-system
// model driver that couples the ice solver into its time loop, or a runtime
// that forbids cudaMalloc/cudaFree after initialisation because those calls
// can synchronise the device and fragment its pool.  Such a caller cannot
// create a glide_handle (which allocates the hierarchy arena), but can still
// evaluate the coupled residual of one level on arrays it already owns.
//
// The only scratch the computation needs -- three partial sums of squares per
// 16 x 16 tile -- lives in the file-scope device array below, so this entry
// point calls no allocating routine at all.  Its size bounds the grid:
// kNoAllocMaxTiles tiles, i.e. up to 65,536 tiles of 16 x 16 cells
// (4096 x 4096 cells, for example), 1.5 MiB per device, held by every GPU that
// loads the library until the process exits.  Independently, a grid has at
// most 65,535 rows.
#include <cuda_runtime.h>

#include <string>

#include "glide_b200.h"
#include "forward_kernels.cuh"

namespace glide {
namespace noalloc {

constexpr long long kNoAllocMaxTiles = 65536;
constexpr long long kNoAllocMaxRows = 65535;

// 3 partial sums per tile; every call rewrites each slot it later reads, so
// nothing needs clearing between calls.  Calls that overlap on the GPU
// (different streams, or concurrent host threads) share this array and race.
static __device__ __align__(256) double g_tile_sums[3 * kNoAllocMaxTiles];

static thread_local std::string t_err;

// Device address of g_tile_sums in the CUDA context current on this thread.
// In host code the symbol itself is only a host-side stand-in, so every call
// looks the address up again: the array belongs to the module loaded in a
// context, not to a device ordinal, and a cached pointer would go stale after
// cudaDeviceReset or point into another context when the host switches
// driver-API contexts on one device.  The lookup allocates nothing.  The first
// lookup in a context loads the module (and with it this array), which is why
// the first call on a device should come before any stream capture.
static int scratch_address(double** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_tile_sums);
    if (e != cudaSuccess || !p) {
        t_err = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
        return GLIDE_ERR_CUDA;
    }
    *out = static_cast<double*>(p);
    return GLIDE_OK;
}

// Fixed-order reduction of the tile sums into norms[0..3] (|r_u|, |r_v|,
// |r_H| and their combined norm).
__global__ void __launch_bounds__(1024) k_noalloc_norms(const double* sums, int ntiles, double* norms) {
    __shared__ double ws[3][32];
    const int t = threadIdx.x, l = t & 31, w = t >> 5;
    double s[3] = {0, 0, 0};
    for (int b = t; b < ntiles; b += 1024)
        for (int q = 0; q < 3; ++q) s[q] += sums[size_t(b) * 3 + q];
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
            norms[0] = sqrt(s[0]);
            norms[1] = sqrt(s[1]);
            norms[2] = sqrt(s[2]);
            norms[3] = sqrt(s[0] + s[1] + s[2]);
        }
    }
}

}  // namespace noalloc
}  // namespace glide

using namespace glide;

extern "C" const char* glide_noalloc_last_error(void) { return noalloc::t_err.c_str(); }

extern "C" int glide_residual_norms_noalloc(int ny, int nx, double dx, double dt, const glide_phys* phys,
                                            const double* u, int ld_u, const double* v, int ld_v,
                                            const double* H, double* phi, const double* mask,
                                            const double* f_u, const double* f_v, const double* f_H,
                                            const double* bed, const double* B, const double* beta,
                                            const double* gamma, int ld_c, int flags, double* r_u,
                                            double* r_v, double* r_H, double* norms, void* stream) {
    using noalloc::t_err;
    if (!phys || !u || !v || !H || !phi || !mask || !bed || !B || !beta || !gamma || !r_u || !r_v || !r_H ||
        !norms) {
        t_err = "null argument";
        return GLIDE_ERR_ARG;
    }
    if (!(flags & GLIDE_OPERATOR_ONLY) && (!f_u || !f_v || !f_H)) {
        t_err = "forcing arrays are required unless GLIDE_OPERATOR_ONLY is set";
        return GLIDE_ERR_ARG;
    }
    // All size arithmetic in 64 bits, so that nx or ny near INT_MAX cannot
    // wrap around and slip past the checks.
    const long long nyl = ny, nxl = nx;
    if (nyl < 2 || nxl < 2 || !(dx > 0) || !(dt > 0) || (long long)ld_u < nxl + 1 || (long long)ld_v < nxl ||
        (long long)ld_c < nxl) {
        t_err = "bad sizes: need ny, nx >= 2, dx, dt > 0, ld_u >= nx + 1, ld_v >= nx, ld_c >= nx";
        return GLIDE_ERR_SHAPE;
    }
    // The grounded-fraction launch puts one grid row per block row, and a
    // grid's y extent is at most 65,535.
    if (nyl > noalloc::kNoAllocMaxRows) {
        t_err = "grid too tall for the no-allocation residual: at most " +
                std::to_string(noalloc::kNoAllocMaxRows) + " rows";
        return GLIDE_ERR_SHAPE;
    }
    const long long tiles_x = (nxl + kTile - 1) / kTile, tiles_y = (nyl + kTile - 1) / kTile;
    if (tiles_x * tiles_y > noalloc::kNoAllocMaxTiles) {
        t_err = "grid too large for the no-allocation residual: at most " +
                std::to_string(noalloc::kNoAllocMaxTiles) + " tiles of 16 x 16 cells (e.g. 4096 x 4096 cells)";
        return GLIDE_ERR_SHAPE;
    }
    double* sums = nullptr;
    int rc = noalloc::scratch_address(&sums);
    if (rc != GLIDE_OK) return rc;

    auto arr = [&](const double* p, int rows, int cols, int ld) {
        Arr<double> a;
        a.p = const_cast<double*>(p);
        a.rows = rows;
        a.cols = cols;
        a.pitch = ld;
        return a;
    };
    const bool op_only = (flags & GLIDE_OPERATOR_ONLY) != 0;
    ResidualArgs<double> a;
    a.u = arr(u, ny, nx + 1, ld_u);
    a.v = arr(v, ny + 1, nx, ld_v);
    a.H = arr(H, ny, nx, ld_c);
    a.phi = arr(phi, ny, nx, ld_c);
    a.mask = arr(mask, ny, nx, ld_c);
    a.bed = arr(bed, ny, nx, ld_c);
    a.B = arr(B, ny, nx, ld_c);
    a.beta = arr(beta, ny, nx, ld_c);
    a.gamma = arr(gamma, ny, nx, ld_c);
    a.f_u = op_only ? Arr<double>() : arr(f_u, ny, nx + 1, ld_u);
    a.f_v = op_only ? Arr<double>() : arr(f_v, ny + 1, nx, ld_v);
    a.f_H = op_only ? Arr<double>() : arr(f_H, ny, nx, ld_c);
    a.o_u = arr(r_u, ny, nx + 1, ld_u);
    a.o_v = arr(r_v, ny + 1, nx, ld_v);
    a.o_H = arr(r_H, ny, nx, ld_c);
    a.partial = sums;
    Phys p{phys->n, phys->eps_reg, phys->flotation_reg_driving, phys->m, phys->u_reg, phys->water_drag,
           phys->flotation_reg_sliding, phys->calving_rate, phys->flotation_reg_calving, phys->thklim};
    a.p = PhysR<double>(p, dx, dt, (flags & GLIDE_FREEZE_CALVING) ? 0.0 : phys->calving_rate);
    a.ny = ny;
    a.nx = nx;
    a.use_forcing = op_only ? 0 : 1;
    a.use_mask = (flags & GLIDE_USE_MASK) ? 1 : 0;
    a.active_set = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    if (!(flags & GLIDE_FREEZE_PHI)) {
        // grounded fraction from H and bed first, as glide_residual does
        k_grounded<double><<<dim3((nx + 255) / 256, ny), 256, 0, s>>>(a.phi, a.H, a.bed, phys->flotation_reg_driving,
                                                                     0.0, ny, nx);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        // caller-owned arrays: the tiles are staged with clamped scalar loads
        BoxMaps<7> maps;
        maps.use = 0;
        a.err = nullptr;
        k_residual<double><<<dim3(unsigned(tiles_x), unsigned(tiles_y)), 256, 0, s>>>(a, maps);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        noalloc::k_noalloc_norms<<<1, 1024, 0, s>>>(sums, int(tiles_x * tiles_y), norms);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        t_err = std::string("kernel launch: ") + cudaGetErrorString(e);
        return GLIDE_ERR_CUDA;
    }
    return GLIDE_OK;
}
