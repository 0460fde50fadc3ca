// io.cu -- device packing of VTK ImageData (VTI) appended data
// (glide/io.py:23-184 write_vti of JacobDowns/glide).
//
// The reference copies every array of a snapshot to the host, casts it to
// binary32, flips it along y, reorders 3-D arrays x-fastest, interleaves
// vector components and writes each array as a uint32 byte count followed
// by its values.  Here one launch reads every array where it lives in HBM
// and writes that whole block into one device buffer; the host then copies
// one contiguous block and writes it after the XML header.  Face arrays are
// averaged to cell centres on the fly (Field.to_cell, glide/field.py:86-107)
// in their own precision, as the reference computes them, so no cell copy
// is materialised.  Layer-major 3-D arrays (level k outermost) are read
// with unit stride along x: every warp reads and writes contiguous runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "glide_b200.h"
#include "glide_io.h"

namespace glide {
namespace io {

static thread_local std::string t_err;

struct Fail {
    int code;
};

[[noreturn]] static void fail(int code, const std::string& msg) {
    t_err = msg;
    throw Fail{code};
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

struct Comp {
    const void* p;
    int f64, kind;
    long long si, sj, sk;
};

// Every array of one snapshot: components, count and byte offset of its
// count word in the output block.
struct Pack {
    Comp c[GLIDE_VTI_MAX_ARRAYS][3];
    int nc[GLIDE_VTI_MAX_ARRAYS];
    unsigned long long off[GLIDE_VTI_MAX_ARRAYS];
    unsigned int count[GLIDE_VTI_MAX_ARRAYS];
};

constexpr int kPackThreads = 256;
constexpr long long kMaxRowBlocks = 4096;

// A component's value at offset e of its array (the point's own element),
// rounded to binary32.
template <class T>
__device__ __forceinline__ float point_value(const T* a, int kind, long long si, long long sj) {
    T x;
    if (kind == GLIDE_VTI_XFACE) x = T(0.5) * (a[sj] + a[0]);
    else if (kind == GLIDE_VTI_YFACE) x = T(0.5) * (a[si] + a[0]);
    else x = a[0];
    return float(x);
}

__device__ __forceinline__ float comp_value(const Comp& c, const void* row, int j) {
    return c.f64 ? point_value(static_cast<const double*>(row) + j * c.sj, c.kind, c.si, c.sj)
                 : point_value(static_cast<const float*>(row) + j * c.sj, c.kind, c.si, c.sj);
}

__device__ __forceinline__ const void* comp_row(const Comp& c, long long k, int i) {
    const long long e = k * c.sk + i * c.si;
    return c.f64 ? static_cast<const void*>(static_cast<const double*>(c.p) + e)
                 : static_cast<const void*>(static_cast<const float*>(c.p) + e);
}

// blockIdx.y: array; blockIdx.x strides the output rows (z outer, y inner);
// threads stride x.  The array's descriptors are copied to registers once
// per block and each row's start is formed once per row, so the inner loop
// is an address step, a load (two for face fields), a conversion and a
// store; 32 registers keep 8 blocks (64 warps) resident per SM.
__global__ void __launch_bounds__(kPackThreads, 8) k_vti_pack(const __grid_constant__ Pack P, int ny, int nx,
                                                           int nz, int flip, unsigned char* dst) {
    const int a = blockIdx.y;
    const int nc = P.nc[a];
    const Comp c0 = P.c[a][0], c1 = P.c[a][1], c2 = P.c[a][2];
    unsigned char* base = dst + P.off[a];
    if (blockIdx.x == 0 && threadIdx.x == 0) *reinterpret_cast<unsigned int*>(base) = P.count[a];
    float* out = reinterpret_cast<float*>(base + 4);
    const long long rows = (long long)ny * nz;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        const long long k = r / ny;
        const int row = int(r - k * ny);
        const int i = flip ? ny - 1 - row : row;
        float* o = out + r * nx * nc;
        const void* r0 = comp_row(c0, k, i);
        if (nc == 1) {
            for (int j = threadIdx.x; j < nx; j += blockDim.x) o[j] = comp_value(c0, r0, j);
            continue;
        }
        const void* r1 = comp_row(c1, k, i);
        const void* r2 = nc > 2 ? comp_row(c2, k, i) : nullptr;
        for (int j = threadIdx.x; j < nx; j += blockDim.x) {
            o[j * nc] = comp_value(c0, r0, j);
            o[j * nc + 1] = comp_value(c1, r1, j);
            if (nc > 2) o[j * nc + 2] = comp_value(c2, r2, j);
        }
    }
}

}  // namespace io
}  // namespace glide

using namespace glide::io;

extern "C" {

const char* glide_io_last_error(void) { return t_err.c_str(); }

int glide_vti_pack(int ny, int nx, int nz, int flip_y, const glide_vti_array* arrays, int n_arrays, void* dst,
                   size_t capacity, size_t* bytes, void* stream) {
    return guarded([&] {
        if (ny < 1 || nx < 1 || nz < 1) fail(GLIDE_ERR_SHAPE, "ny, nx and nz must be at least 1");
        if (!arrays || n_arrays < 1 || n_arrays > GLIDE_VTI_MAX_ARRAYS)
            fail(GLIDE_ERR_ARG, "n_arrays must lie in [1, GLIDE_VTI_MAX_ARRAYS]");
        if (!bytes) fail(GLIDE_ERR_ARG, "null bytes pointer");
        Pack P{};
        const unsigned long long points = (unsigned long long)ny * nx * nz;
        unsigned long long off = 0;
        for (int a = 0; a < n_arrays; ++a) {
            const glide_vti_array& A = arrays[a];
            if (A.n_components < 1 || A.n_components > 3) fail(GLIDE_ERR_ARG, "n_components must be 1, 2 or 3");
            const unsigned long long nb = points * (unsigned long long)A.n_components * 4ull;
            if (nb >= (1ull << 32))
                fail(GLIDE_ERR_SHAPE, "an array of 2^32 bytes or more does not fit the 32-bit count word");
            for (int q = 0; q < A.n_components; ++q) {
                const glide_vti_component& c = A.comp[q];
                if (dst && !c.data) fail(GLIDE_ERR_ARG, "null component data");
                if (c.dtype != GLIDE_F64 && c.dtype != GLIDE_F32)
                    fail(GLIDE_ERR_ARG, "component dtype must be GLIDE_F64 or GLIDE_F32");
                if (c.kind != GLIDE_VTI_PLAIN && c.kind != GLIDE_VTI_XFACE && c.kind != GLIDE_VTI_YFACE)
                    fail(GLIDE_ERR_ARG, "unknown component kind");
                P.c[a][q] = Comp{c.data, c.dtype == GLIDE_F64, c.kind, c.stride_i, c.stride_j, c.stride_k};
            }
            P.nc[a] = A.n_components;
            P.off[a] = off;
            P.count[a] = unsigned(nb);
            off += 4ull + nb;
        }
        *bytes = size_t(off);
        if (!dst) return;
        if (capacity < off) fail(GLIDE_ERR_ARG, "destination smaller than the appended-data block");
        if (reinterpret_cast<uintptr_t>(dst) % 4) fail(GLIDE_ERR_ARG, "destination must be 4-byte aligned");
        const long long rows = (long long)ny * nz;
        const dim3 grid(unsigned(std::min(rows, kMaxRowBlocks)), unsigned(n_arrays));
        k_vti_pack<<<grid, kPackThreads, 0, static_cast<cudaStream_t>(stream)>>>(
            P, ny, nx, nz, flip_y != 0, static_cast<unsigned char*>(dst));
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) fail(GLIDE_ERR_CUDA, std::string("vti pack launch: ") + cudaGetErrorString(e));
    });
}

}  // extern "C"
