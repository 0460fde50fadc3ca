"""VTK ImageData (VTI) snapshots and their PVD manifest: write_vti and
VTIWriter of glide/io.py (:18-390, JacobDowns/glide), with the array work on
the GPU.

The reference copies each array to the host, casts it to binary32, flips it
along y, reorders 3-D arrays x-fastest and interleaves vector components,
all in NumPy.  Here one kernel (glide_vti_pack, include/glide_io.h) reads
every array of a snapshot where it lives in HBM and writes the file's whole
appended-data block into one device buffer.  It averages face fields to
cell centres on the fly (Field.to_cell, glide/field.py:86-107), so no cell
copy is made.  One copy brings the block to pinned host memory, and the host
writes the XML header and the block.  The header is built with the same
xml.etree calls as the reference, so the files are byte-for-byte the
reference's.

VTIWriter(background=True) overlaps the copy and the file write with the
solver: the pack runs on the current stream, the copy on a side stream, and
a host thread writes the file; `flush()` waits for every pending file.
"""
from __future__ import annotations

import ctypes
import threading
import xml.etree.ElementTree as ET
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any, Mapping
from xml.dom import minidom

import numpy as np
import torch

from . import _lib
from ._lib import GlideError

_APPENDED_OPEN = b'  <AppendedData encoding="raw">\n   _'
_APPENDED_CLOSE = b"\n  </AppendedData>\n</VTKFile>\n"


def _pretty_xml(element) -> str:
    """Indented XML text of an element (the reference's PVD formatting)."""
    return minidom.parseString(ET.tostring(element)).toprettyxml(indent="  ")


def _io_call(name, *args):
    lib = _lib.load()
    code = getattr(lib, name)(*args)
    if code != _lib.GLIDE_OK:
        msg = lib.glide_io_last_error()
        raise GlideError(code, msg.decode() if msg else "")


# ----------------------------------------------------------------- values
class _Comp:
    """One array read by the pack kernel: a CUDA tensor and how to read it
    (plain, or u / v faces averaged to cell centres)."""

    def __init__(self, t: torch.Tensor, kind: int):
        if t.dtype not in (torch.float32, torch.float64):
            t = t.to(torch.float64)
        self.t = t
        self.kind = kind
        s = tuple(t.shape)
        if kind == _lib.VTI_XFACE:
            s = (s[0], s[1] - 1) + s[2:]
        elif kind == _lib.VTI_YFACE:
            s = (s[0] - 1,) + s[1:]
        self.shape = s

    @property
    def ndim(self) -> int:
        return len(self.shape)

    def descriptor(self) -> _lib.VtiComponent:
        t = self.t
        st = t.stride()
        return _lib.VtiComponent(t.data_ptr(), _lib.GLIDE_F64 if t.dtype == torch.float64 else _lib.GLIDE_F32,
                                 self.kind, st[0], st[1], st[2] if t.dim() == 3 else 0)


def _tensor(a) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a if a.is_cuda else a.cuda()
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # views with negative strides included


def _entity(value) -> str | None:
    ge = getattr(value, "grid_entity", None)
    return None if ge is None else str(getattr(ge, "value", ge))


def _component(value) -> _Comp:
    """Resolve a field value as the reference's _coerce_*_value does: a
    callable is evaluated now; a field object contributes its cell-centred
    data (face fields averaged by the kernel); arrays are taken as they are."""
    if callable(value) and not hasattr(value, "data"):
        value = value()
    if isinstance(value, (torch.Tensor, np.ndarray)):
        return _Comp(_tensor(value), _lib.VTI_PLAIN)
    ent = _entity(value)
    if ent is not None and hasattr(value, "data"):
        kind = {"vertical_facet": _lib.VTI_XFACE, "horizontal_facet": _lib.VTI_YFACE}.get(ent, _lib.VTI_PLAIN)
        t = _tensor(value.data)
        if kind != _lib.VTI_PLAIN and t.dim() != 2:
            raise ValueError(f"face field of shape {tuple(t.shape)}: only 2-D face fields average to cells")
        return _Comp(t, kind)
    if hasattr(value, "to_cell"):
        value = value.to_cell()
        return _Comp(_tensor(getattr(value, "data", value)), _lib.VTI_PLAIN)
    if hasattr(value, "data"):
        return _Comp(_tensor(value.data), _lib.VTI_PLAIN)
    return _Comp(_tensor(value), _lib.VTI_PLAIN)


# ----------------------------------------------------------------- header
def _vti_header(scalars, vectors, dims, is_3d, dx, dy, dz, origin, time_value) -> bytes:
    """XML of write_vti (glide/io.py:106-165) up to, not including, the
    closing </VTKFile>; array offsets count the 4-byte size words."""
    ny, nx, nz = dims
    if len(origin) == 2:
        origin3 = (float(origin[0]), float(origin[1]), 0.0)
    else:
        origin3 = (float(origin[0]), float(origin[1]), float(origin[2]))
    extent = f"0 {nx-1} 0 {ny-1} 0 {nz-1}"
    spacing = f"{dx} {dy} {dz if is_3d else 1.0}"
    root = ET.Element("VTKFile", type="ImageData", version="1.0", byte_order="LittleEndian")
    img = ET.SubElement(root, "ImageData", WholeExtent=extent,
                        Origin=f"{origin3[0]} {origin3[1]} {origin3[2]}", Spacing=spacing)
    piece = ET.SubElement(img, "Piece", Extent=extent)
    if time_value is not None:
        fd = ET.SubElement(piece, "FieldData")
        da = ET.SubElement(fd, "DataArray", type="Float32", Name="TimeValue", NumberOfComponents="1",
                           format="ascii")
        da.text = f"\n{float(time_value)}\n"
    pd_attrs = {}
    if scalars:
        pd_attrs["Scalars"] = next(iter(scalars))
    for name, comps in vectors.items():
        if len(comps) == 3:
            pd_attrs["Vectors"] = name
            break
    pd = ET.SubElement(piece, "PointData", **pd_attrs)
    npts = nx * ny * nz
    offset = 0
    for name in scalars:
        ET.SubElement(pd, "DataArray", type="Float32", Name=name, NumberOfComponents="1", format="appended",
                      offset=str(offset))
        offset += 4 * npts + 4
    for name, comps in vectors.items():
        ET.SubElement(pd, "DataArray", type="Float32", Name=name, NumberOfComponents=str(len(comps)),
                      format="appended", offset=str(offset))
        offset += 4 * npts * len(comps) + 4
    text = ET.tostring(root, encoding="utf-8", xml_declaration=True).decode("utf-8")
    for tail in ("</VTKFile>", "</VTKFile>\n"):
        if text.endswith(tail):
            text = text[: -len(tail)]
            break
    return text.encode("utf-8")


# ----------------------------------------------------------------- a snapshot
class _Snapshot:
    """Resolved arrays of one write_vti call and its header."""

    def __init__(self, data: Mapping[str, Any], dx, dy, dz, origin, time_value, flip_y):
        scalars: dict[str, _Comp] = {}
        vectors: dict[str, list[_Comp]] = {}
        for name, value in data.items():
            if isinstance(value, (list, tuple)):
                vectors[name] = [_component(c) for c in value]
            else:
                scalars[name] = _component(value)
        if not scalars and not vectors:
            raise ValueError("write_vti needs at least one field")
        first = next(iter(scalars.values())) if scalars else next(iter(vectors.values()))[0]
        if first.ndim == 2:
            is_3d = False
            ny, nx = first.shape
            nz = 1
        elif first.ndim == 3:
            is_3d = True
            ny, nx, nz = first.shape
            if dz is None:
                raise ValueError("dz must be provided for 3D output (got 3D field with shape "
                                 f"{first.shape})")
            if vectors:
                raise NotImplementedError("Vector fields are only supported in 2D mode.")
        else:
            raise ValueError(f"Field arrays must be 2D or 3D; got shape {first.shape}")
        for name, c in scalars.items():
            if c.ndim != first.ndim:
                raise ValueError(f"Field '{name}' has shape {c.shape}; expected "
                                 f"{'3D' if is_3d else '2D'} like the first field.")
            if c.shape != first.shape:
                raise ValueError(f"Field '{name}' has shape {c.shape}; expected {first.shape} like the "
                                 "first field.")
        for name, comps in vectors.items():
            if not 1 <= len(comps) <= 3:
                raise ValueError(f"Vector field '{name}' has {len(comps)} components; expected 1 to 3.")
            for c in comps:
                if c.shape != (ny, nx):
                    raise ValueError(f"Vector field '{name}' has a component of shape {c.shape}; expected "
                                     f"{(ny, nx)}.")
        self.dims = (ny, nx, nz)
        self.flip_y = bool(flip_y)
        self.arrays = [[c] for c in scalars.values()] + list(vectors.values())
        self.header = _vti_header(scalars, vectors, self.dims, is_3d, dx, dy, dz, origin, time_value)
        npts = ny * nx * nz
        self.nbytes = sum(4 + 4 * npts * len(a) for a in self.arrays)

    def pack(self, dst: torch.Tensor, stream: torch.cuda.Stream) -> None:
        """Launch the pack kernel(s) into the device buffer dst on stream."""
        ny, nx, nz = self.dims
        base = dst.data_ptr()
        off = 0
        done = ctypes.c_size_t()
        for g in range(0, len(self.arrays), _lib.VTI_MAX_ARRAYS):
            group = self.arrays[g:g + _lib.VTI_MAX_ARRAYS]
            desc = (_lib.VtiArray * len(group))()
            for a, comps in zip(desc, group):
                a.n_components = len(comps)
                for q, c in enumerate(comps):
                    a.comp[q] = c.descriptor()
            _io_call("glide_vti_pack", ny, nx, nz, int(self.flip_y), desc, len(group),
                     ctypes.c_void_p(base + off), ctypes.c_size_t(self.nbytes - off), ctypes.byref(done),
                     ctypes.c_void_p(stream.cuda_stream))
            off += done.value
        assert off == self.nbytes


def _write_file(path: Path, header: bytes, payload) -> None:
    with open(path, "wb") as f:
        f.write(header)
        f.write(_APPENDED_OPEN)
        f.write(payload)
        f.write(_APPENDED_CLOSE)


class _Staging:
    """A device buffer and a pinned host buffer, grown on demand."""

    def __init__(self):
        self.dev = None
        self.host = None

    def get(self, n: int):
        if self.dev is None or self.dev.numel() < n:
            self.dev = torch.empty(n, dtype=torch.uint8, device="cuda")
            self.host = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        return self.dev, self.host


_sync_staging = threading.local()


def write_vti(filename, data, dx, dy=None, dz=None, origin=(0.0, 0.0), time_value=None, flip_y=True):
    """Write fields to a VTI (VTK ImageData) file with raw appended binary32
    data: glide/io.py:23-184.

    data maps names to 2-D (ny, nx) or 3-D (ny, nx, nz) arrays (CUDA or CPU
    tensors, NumPy arrays), field objects (face fields are averaged to cell
    centres) or lists of 2-D components (vectors).  3-D output needs dz and
    takes no vectors.  origin is (x, y) or (x, y, z).  flip_y writes row
    ny - 1 first (image rows to VTK's upward y).  Returns when the file is
    written.  Each host thread keeps one device and one pinned host staging
    buffer, grown to the largest snapshot it has written, for reuse by later
    calls; release_staging() frees them."""
    if dy is None:
        dy = dx
    Path(filename).parent.mkdir(parents=True, exist_ok=True)
    snap = _Snapshot(data, dx, dy, dz, origin, time_value, flip_y)
    st = getattr(_sync_staging, "buf", None)
    if st is None:
        st = _sync_staging.buf = _Staging()
    dev, host = st.get(snap.nbytes)
    stream = torch.cuda.current_stream()
    snap.pack(dev, stream)
    host[: snap.nbytes].copy_(dev[: snap.nbytes], non_blocking=True)
    stream.synchronize()
    _write_file(Path(filename), snap.header, memoryview(host.numpy())[: snap.nbytes])


def release_staging() -> None:
    """Free this thread's write_vti staging buffers (device and pinned host)."""
    _sync_staging.buf = None


class _Background:
    """Two staging slots, a copy stream and one writer thread."""

    def __init__(self):
        self.slots = [_Staging(), _Staging()]
        self.busy: list[Future | None] = [None, None]
        self.next = 0
        self.copy_stream = torch.cuda.Stream()
        self.pool = ThreadPoolExecutor(max_workers=1, thread_name_prefix="vti-writer")

    def submit(self, path: Path, snap: _Snapshot) -> None:
        s = self.next
        self.next ^= 1
        if self.busy[s] is not None:
            self.busy[s].result()
        dev, host = self.slots[s].get(snap.nbytes)
        compute = torch.cuda.current_stream()
        snap.pack(dev, compute)
        packed = torch.cuda.Event()
        packed.record(compute)
        copied = torch.cuda.Event()
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(packed)
            host[: snap.nbytes].copy_(dev[: snap.nbytes], non_blocking=True)
            copied.record(self.copy_stream)
        n, header = snap.nbytes, snap.header

        def job():
            copied.synchronize()
            _write_file(path, header, memoryview(host.numpy())[:n])

        self.busy[s] = self.pool.submit(job)

    def flush(self) -> None:
        for f in self.busy:
            if f is not None:
                f.result()


@dataclass
class VTIWriter:
    """Static and time-dependent VTI output with a PVD manifest
    (glide/io.py:187-390): configure static_fields and dynamic_fields, call
    initialize once, then append for each snapshot and write_pvd for the
    manifest.  Values are fields (face fields averaged to cell centres),
    arrays, callables evaluated at write time, or lists of those (vectors).
    All fields of one writer are either 2-D or 3-D (3-D needs dz).

    background=True (no counterpart in the reference): a call returns once
    the snapshot is packed on the GPU; the copy to the host and the file
    write run behind the caller, two snapshots deep.  flush() (also called by
    write_pvd) waits for them."""

    out_dir: str | Path
    static_fields: Mapping[str, Any] = field(default_factory=dict)
    dynamic_fields: Mapping[str, Any] = field(default_factory=dict)
    base: str = "output"
    dx: float = 1.0
    dy: float | None = None
    dz: float | None = None
    origin: tuple = (0.0, 0.0)
    flip_y: bool = True
    background: bool = False

    _step_idx: int = field(default=0, init=False, repr=False)
    _static_written: bool = field(default=False, init=False, repr=False)
    records: list[tuple[float, str]] = field(default_factory=list, init=False, repr=False)
    _bg: _Background | None = field(default=None, init=False, repr=False)

    def __post_init__(self) -> None:
        self.out_dir = Path(self.out_dir)
        self.out_dir.mkdir(parents=True, exist_ok=True)
        if self.dy is None:
            self.dy = self.dx

    # public high-level API
    def initialize(self, grid: Any, *, overwrite: bool = False, write_dynamic_initial: bool = False,
                   time: Any | None = None) -> None:
        """Optionally clear earlier output, write the static fields and an
        initial dynamic snapshot."""
        if overwrite:
            self.flush()
            for path in self.out_dir.glob(f"{self.base}_*.vti"):
                path.unlink()
            pvd_path = self.out_dir / f"{self.base}.pvd"
            if pvd_path.exists():
                pvd_path.unlink()
            self.records.clear()
            self._step_idx = 0
            self._static_written = False
        if self.static_fields:
            self.write_static(grid, overwrite=overwrite)
        if write_dynamic_initial:
            if time is None:
                raise ValueError("Argument `time` must be provided when write_dynamic_initial=True.")
            self.append(grid, time=time)

    def append(self, grid: Any, *, time: Any) -> Path:
        """Append one dynamic snapshot at the given time."""
        if not self.dynamic_fields:
            raise ValueError("No dynamic fields were configured for this writer.")
        return self.append_dynamic(grid, time=time)

    # lower-level API
    def write_static(self, grid: Any, *, overwrite: bool = False) -> Path | None:
        """Write the static fields once to {base}_static.vti."""
        if not self.static_fields:
            return None
        fpath = self.out_dir / f"{self.base}_static.vti"
        if self._static_written and not overwrite:
            return fpath
        self._write(fpath, self.static_fields, None)
        self._static_written = True
        return fpath

    def append_dynamic(self, grid: Any, *, time: Any) -> Path:
        """Append one time slice of the dynamic fields."""
        fpath = self.write_step(self._step_idx, time, self.dynamic_fields)
        self._step_idx += 1
        return fpath

    def write_step(self, step_idx: int, time_value: Any, data: Mapping[str, Any]) -> Path:
        """Write a time step to {base}_{step_idx:04d}.vti and record it."""
        fname = f"{self.base}_{step_idx:04d}.vti"
        fpath = self.out_dir / fname
        self._write(fpath, data, time_value)
        self.records.append((float(time_value), fname))
        return fpath

    def write_pvd(self, pvd_name: str | None = None) -> Path:
        """Write the PVD manifest of the recorded steps (after every pending
        snapshot file is on disk)."""
        self.flush()
        if pvd_name is None:
            pvd_name = f"{self.base}.pvd"
        root = ET.Element("VTKFile", type="Collection", version="0.1", byte_order="LittleEndian")
        coll = ET.SubElement(root, "Collection")
        for t, fname in self.records:
            ET.SubElement(coll, "DataSet", timestep=str(t), group="", part="0", file=str(fname))
        with open(self.out_dir / pvd_name, "w") as f:
            f.write(_pretty_xml(root))
        return self.out_dir / pvd_name

    def flush(self) -> None:
        """Wait until every snapshot handed to the background writer is on disk."""
        if self._bg is not None:
            self._bg.flush()

    def _write(self, fpath: Path, fields: Mapping[str, Any], time_value) -> None:
        if not self.background:
            write_vti(fpath, dict(fields), self.dx, dy=self.dy, dz=self.dz, origin=self.origin,
                      time_value=time_value, flip_y=self.flip_y)
            return
        if self._bg is None:
            self._bg = _Background()
        snap = _Snapshot(dict(fields), self.dx, self.dy, self.dz, self.origin, time_value, self.flip_y)
        self._bg.submit(fpath, snap)
