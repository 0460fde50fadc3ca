/* glide_io.h -- C ABI of the device-side packing of VTK ImageData (VTI)
 * output: the appended-data block of glide/io.py write_vti (:23-184 of
 * JacobDowns/glide), produced from device arrays in one kernel launch.
 *
 * Reference interface each entry point replaces (paths inside the
 * JacobDowns/glide project):
 *   glide_vti_pack   the array part of write_vti (glide/io.py:60-75 host copy,
 *                    binary32 cast and y flip; :137-163 x-fastest ordering and
 *                    vector interleave; :174-182 the uint32 byte count before
 *                    each array), with Field.to_cell (glide/field.py:86-107)
 *                    applied to face arrays on the fly
 *   glide_io_last_error   message of the last failure on this thread
 *
 * The XML header, the file and the PVD manifest are written by the host
 * (glide_b200/io.py); this call produces the bytes that follow the '_'
 * marker of <AppendedData encoding="raw">.
 */
#ifndef GLIDE_IO_H
#define GLIDE_IO_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GLIDE_VTI_MAX_ARRAYS 16

/* How a component is read at output point (i, j, k):
 *   GLIDE_VTI_PLAIN   a[i, j, k]
 *   GLIDE_VTI_XFACE   0.5 (a[i, j+1] + a[i, j])   u faces to cell centres
 *   GLIDE_VTI_YFACE   0.5 (a[i+1, j] + a[i, j])   v faces to cell centres
 * the sum and the halving in the array's own precision, then rounded to
 * binary32 (to nearest, ties to even). */
#define GLIDE_VTI_PLAIN 0
#define GLIDE_VTI_XFACE 1
#define GLIDE_VTI_YFACE 2

/* One component: a device array of dtype GLIDE_F64 (0) or GLIDE_F32 (1)
 * (glide_b200.h), element strides of row i, column j and level k (k is 0
 * for 2-D output). */
typedef struct {
    const void* data;
    int dtype;
    int kind;
    long long stride_i, stride_j, stride_k;
} glide_vti_component;

/* One DataArray: 1 component (scalar) or 2 / 3 (vector, interleaved). */
typedef struct {
    int n_components;
    glide_vti_component comp[3];
} glide_vti_array;

/* Writes, for each of the n_arrays arrays in order, the uint32 byte count
 * of its values followed by ny * nx * nz * n_components binary32 values,
 * x fastest, then y (row ny - 1 - i first when flip_y), then z, into the
 * device buffer dst (capacity bytes, 4-byte aligned).  *bytes receives the
 * block's size; with dst == NULL nothing else happens (a size query).
 * Launches one kernel on `stream` and does not synchronise.  Errors:
 * GLIDE_ERR_ARG for a bad count, dtype, kind or pointer, or a capacity
 * below the block's size; GLIDE_ERR_SHAPE for a non-positive extent or an
 * array whose values take 2^32 bytes or more (the count word is 32 bits). */
int glide_vti_pack(int ny, int nx, int nz, int flip_y, const glide_vti_array* arrays, int n_arrays,
                   void* dst, size_t capacity, size_t* bytes, void* stream);
const char* glide_io_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GLIDE_IO_H */
