"""NumPy restatement of the reference's VTI writer (test infrastructure only).

Follows write_vti of glide/io.py (JacobDowns/glide) :23-184: binary32 cast
(:64-73), y flip (:67-73), dimensionality checks (:76-101), the ImageData /
Piece / FieldData / PointData header (:106-133), x-fastest ordering of 3-D
arrays (:136-145), vector interleave (:153-163) and the raw appended block
with a uint32 byte count before every array (:165-182); the PVD manifest of
VTIWriter.write_pvd (:330-353); Field.to_cell (glide/field.py:86-107) for
face arrays.  The header is written out as text here, independently of
the xml.etree calls the product uses.  Pinned against files written by the
reference's own writer (tests/golden/vti/, tests/golden/make_vti_golden.py).
Only tests and the bench's CPU baseline use it.
"""
from __future__ import annotations

import numpy as np


def to_cell(a: np.ndarray, entity: str) -> np.ndarray:
    """Field.to_cell: u faces (ny, nx+1) or v faces (ny+1, nx) averaged to
    cells in the array's own precision."""
    if entity == "vertical_facet":
        return 0.5 * (a[:, 1:] + a[:, :-1])
    if entity == "horizontal_facet":
        return 0.5 * (a[1:] + a[:-1])
    return a


def vti_bytes(data: dict, dx, dy=None, dz=None, origin=(0.0, 0.0), time_value=None, flip_y=True) -> bytes:
    """The bytes write_vti writes for `data` (name -> array, or list of 2-D
    arrays for a vector)."""
    if dy is None:
        dy = dx
    scalars, vectors = {}, {}
    for name, value in data.items():
        if isinstance(value, list):
            comps = [np.asarray(c).astype(np.float32) for c in value]
            vectors[name] = [np.flip(c, axis=0) for c in comps] if flip_y else comps
        else:
            arr = np.asarray(value).astype(np.float32)
            scalars[name] = np.flip(arr, axis=0) if flip_y else arr
    first = next(iter(scalars.values())) if scalars else next(iter(vectors.values()))[0]
    if first.ndim == 2:
        is_3d = False
        (ny, nx), nz = first.shape, 1
    elif first.ndim == 3:
        is_3d = True
        ny, nx, nz = first.shape
        if dz is None:
            raise ValueError("3-D output needs dz")
        if vectors:
            raise NotImplementedError("vectors are 2-D only")
    else:
        raise ValueError("fields must be 2-D or 3-D")
    for name, arr in scalars.items():
        if arr.ndim != first.ndim:
            raise ValueError(f"field {name} differs in dimension from the first field")
    o = (float(origin[0]), float(origin[1]), float(origin[2]) if len(origin) > 2 else 0.0)
    extent = f"0 {nx - 1} 0 {ny - 1} 0 {nz - 1}"
    spacing = f"{dx} {dy} {dz if is_3d else 1.0}"
    head = ("<?xml version='1.0' encoding='utf-8'?>\n"
            '<VTKFile type="ImageData" version="1.0" byte_order="LittleEndian">'
            f'<ImageData WholeExtent="{extent}" Origin="{o[0]} {o[1]} {o[2]}" Spacing="{spacing}">'
            f'<Piece Extent="{extent}">')
    if time_value is not None:
        head += ('<FieldData><DataArray type="Float32" Name="TimeValue" NumberOfComponents="1" '
                 f'format="ascii">\n{float(time_value)}\n</DataArray></FieldData>')
    attrs = ""
    if scalars:
        attrs += f' Scalars="{next(iter(scalars))}"'
    three = [n for n, c in vectors.items() if len(c) == 3]
    if three:
        attrs += f' Vectors="{three[0]}"'
    head += f"<PointData{attrs}>"
    blocks, offset = [], 0
    for name, arr in scalars.items():
        if arr.ndim == 3:
            arr = arr.transpose(2, 0, 1)
        b = np.ascontiguousarray(arr).tobytes()
        head += (f'<DataArray type="Float32" Name="{name}" NumberOfComponents="1" format="appended" '
                 f'offset="{offset}" />')
        blocks.append(b)
        offset += len(b) + 4
    for name, comps in vectors.items():
        b = np.stack(comps, axis=-1).astype(np.float32).tobytes()
        head += (f'<DataArray type="Float32" Name="{name}" NumberOfComponents="{len(comps)}" '
                 f'format="appended" offset="{offset}" />')
        blocks.append(b)
        offset += len(b) + 4
    head += "</PointData></Piece></ImageData>"
    out = [head.encode("utf-8"), b'  <AppendedData encoding="raw">\n   _']
    for b in blocks:
        out += [np.uint32(len(b)).tobytes(), b]
    out.append(b"\n  </AppendedData>\n</VTKFile>\n")
    return b"".join(out)


def pvd_text(records) -> str:
    """VTIWriter.write_pvd's manifest of (time, file name) records."""
    lines = ['<?xml version="1.0" ?>', '<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">',
             "  <Collection>"]
    for t, fname in records:
        lines.append(f'    <DataSet timestep="{t}" group="" part="0" file="{fname}"/>')
    lines += ["  </Collection>", "</VTKFile>", ""]
    return "\n".join(lines)
