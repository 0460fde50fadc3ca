"""VTI / PVD output (glide/io.py:23-390): the oracle restatement against the
files the reference's own writer produced (tests/golden/vti/, made by
tests/golden/make_vti_golden.py), and the host-side header builder of
glide_b200.io against the same files.  No GPU is used here."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

G = Path(__file__).resolve().parent / "golden" / "vti"


@pytest.fixture(scope="module")
def f():
    with np.load(G / "inputs.npz") as z:
        return {k: z[k] for k in z.files}


def _cells(f):
    from oracle import vti_oracle as vo
    return vo.to_cell(f["u"], "vertical_facet"), vo.to_cell(f["v"], "horizontal_facet")


def cases(f):
    """(golden file, oracle arguments) of every single-file case."""
    u, v = _cells(f)
    return [
        ("scalars_vector2.vti", ({"H": f["H"], "U": [u, v], "B": f["B"]}, 1000.0),
         dict(origin=(100.0, -50.0), time_value=2.5)),
        ("vector3_noflip.vti", ({"W": [f["a"], f["b"], f["c"]], "bed": f["bed"]}, 250.0),
         dict(dy=500.0, flip_y=False)),
        ("volume.vti", ({"E": f["E"], "T": f["T"]}, 2000.0), dict(dz=0.5, origin=(1.0, 2.0, 3.0), time_value=10)),
        ("series/dome_static.vti", ({"bed": f["bed"]}, 1000.0), {}),
        ("series/dome_0000.vti", ({"H": f["H"], "U": [u, v], "Hsq": f["H"] * 2.0}, 1000.0), dict(time_value=0.0)),
        ("series/dome_0001.vti", ({"H": f["H1"], "U": [u, v], "Hsq": f["H1"] * 2.0}, 1000.0),
         dict(time_value=5.0)),
    ]


def test_oracle_matches_reference_files(f):
    from oracle import vti_oracle as vo
    for name, args, kw in cases(f):
        assert vo.vti_bytes(*args, **kw) == (G / name).read_bytes(), name
    assert vo.pvd_text([(0.0, "dome_0000.vti"), (5.0, "dome_0001.vti")]) == (G / "series/dome.pvd").read_text()


def test_oracle_dimension_errors(f):
    from oracle import vti_oracle as vo
    with pytest.raises(ValueError):
        vo.vti_bytes({"E": f["E"]}, 1.0)
    with pytest.raises(NotImplementedError):
        vo.vti_bytes({"E": f["E"], "U": [f["a"], f["c"]]}, 1.0, dz=1.0)
    with pytest.raises(ValueError):
        vo.vti_bytes({"H": f["H"], "E": f["E"]}, 1.0, dz=1.0)


def test_product_header_matches_reference_files(f):
    """glide_b200.io builds the XML part on the host: compare it with every
    golden file up to the appended-data marker."""
    from glide_b200.io import _vti_header
    marker = b'  <AppendedData encoding="raw">'
    for name, (data, dx), kw in cases(f):
        scalars = {k: None for k, val in data.items() if not isinstance(val, list)}
        vectors = {k: val for k, val in data.items() if isinstance(val, list)}
        first = next(iter(data.values()))
        shape = (first[0] if isinstance(first, list) else first).shape
        dims = (shape[0], shape[1], shape[2] if len(shape) == 3 else 1)
        hdr = _vti_header(scalars, vectors, dims, len(shape) == 3, dx, kw.get("dy", dx), kw.get("dz"),
                          kw.get("origin", (0.0, 0.0)), kw.get("time_value"))
        gold = (G / name).read_bytes()
        assert hdr == gold[: gold.index(marker)], name


def test_writer_manifest_and_bookkeeping(tmp_path):
    """VTIWriter's host side (glide/io.py:187-353) without a snapshot: the PVD
    manifest of recorded steps is the reference's file, initialize(overwrite=
    True) clears earlier output and the records, and the argument errors of
    append / initialize are the reference's."""
    from glide_b200.io import VTIWriter
    w = VTIWriter(out_dir=tmp_path, base="dome", dx=1000.0)
    assert w.dy == 1000.0 and w.write_static(None) is None
    w.records += [(0.0, "dome_0000.vti"), (5.0, "dome_0001.vti")]
    w.write_pvd()
    assert (tmp_path / "dome.pvd").read_bytes() == (G / "series" / "dome.pvd").read_bytes()
    (tmp_path / "dome_0000.vti").write_bytes(b"x")
    (tmp_path / "other_0000.vti").write_bytes(b"x")
    w.initialize(None, overwrite=True)
    assert not (tmp_path / "dome_0000.vti").exists() and not (tmp_path / "dome.pvd").exists()
    assert (tmp_path / "other_0000.vti").exists() and w.records == []
    with pytest.raises(ValueError, match="No dynamic fields"):
        w.append(None, time=0.0)
    w2 = VTIWriter(out_dir=tmp_path, dynamic_fields={"H": np.zeros((2, 2))})
    with pytest.raises(ValueError, match="`time` must be provided"):
        w2.initialize(None, write_dynamic_initial=True)


def test_release_staging_without_buffers():
    """release_staging frees this thread's write_vti buffers; with none
    allocated it is a no-op (no GPU touched)."""
    from glide_b200 import io as gio
    gio.release_staging()
    assert getattr(gio._sync_staging, "buf", None) is None


def test_pack_size_query_and_argument_errors_without_gpu():
    """glide_vti_pack through the C ABI with no destination (a size query,
    no device work): the block's byte count, and the argument checks."""
    import ctypes

    from glide_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built")
    lib = _lib.load()
    arrays = (_lib.VtiArray * 3)()
    for a, nc in zip(arrays, (1, 2, 3)):
        a.n_components = nc
        for q in range(nc):
            a.comp[q] = _lib.VtiComponent(None, _lib.GLIDE_F64, _lib.VTI_PLAIN, 5, 1, 0)
    n = ctypes.c_size_t()
    ny, nx, nz = 6, 5, 2
    assert lib.glide_vti_pack(ny, nx, nz, 1, arrays, 3, None, 0, ctypes.byref(n), None) == _lib.GLIDE_OK
    assert n.value == sum(4 + 4 * ny * nx * nz * c for c in (1, 2, 3))
    assert lib.glide_vti_pack(0, nx, nz, 1, arrays, 3, None, 0, ctypes.byref(n), None) == _lib.GLIDE_ERR_SHAPE
    assert lib.glide_vti_pack(ny, nx, nz, 1, arrays, 0, None, 0, ctypes.byref(n), None) == _lib.GLIDE_ERR_ARG
    assert lib.glide_vti_pack(ny, nx, nz, 1, arrays, 17, None, 0, ctypes.byref(n), None) == _lib.GLIDE_ERR_ARG
    assert b"n_arrays" in lib.glide_io_last_error()
    arrays[0].comp[0].dtype = 7
    assert lib.glide_vti_pack(ny, nx, nz, 1, arrays, 3, None, 0, ctypes.byref(n), None) == _lib.GLIDE_ERR_ARG
    arrays[0].comp[0].dtype = _lib.GLIDE_F32
    arrays[0].comp[0].kind = 3
    assert lib.glide_vti_pack(ny, nx, nz, 1, arrays, 3, None, 0, ctypes.byref(n), None) == _lib.GLIDE_ERR_ARG
    arrays[0].comp[0].kind = _lib.VTI_XFACE
    arrays[1].n_components = 4
    assert lib.glide_vti_pack(ny, nx, nz, 1, arrays, 3, None, 0, ctypes.byref(n), None) == _lib.GLIDE_ERR_ARG
    arrays[1].n_components = 2
    # values of 2^32 bytes or more do not fit the 32-bit count word
    assert lib.glide_vti_pack(1 << 15, 1 << 15, 1, 1, arrays, 1, None, 0, ctypes.byref(n), None) == \
        _lib.GLIDE_ERR_SHAPE
