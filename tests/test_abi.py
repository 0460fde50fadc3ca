"""The C-ABI library loads on a host without a GPU and exports every entry
point the public headers declare; the ctypes table binds each of them.
No compute call is made here."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(glide_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def header_defines():
    """Every integer #define GLIDE_* of the public headers."""
    out = {}
    for h in sorted((ROOT / "include").glob("*.h")):
        for name, val in re.findall(r"^#define (GLIDE_\w+) (-?\d+)\b", h.read_text(), flags=re.M):
            out[name] = int(val)
    return out


def python_name(define):
    """The glide_b200._lib constant that mirrors a header define."""
    name = define[len("GLIDE_"):]
    if name.startswith(("ERR_", "F64", "F32", "MIXED")) or name == "OK":
        return "GLIDE_" + name
    if name.startswith("GRAD_") and name.endswith("_BIT"):
        return name[:-len("_BIT")]
    return name


def test_python_constants_match_the_headers():
    """Error codes, precisions, flags, tuning keys (solver, group, enthalpy),
    term bits and VTI kinds as the Python layer passes them through the ABI
    equal the headers' values, and none of the keys lacks a mirror."""
    from glide_b200 import _lib
    defines = header_defines()
    must = [d for d in defines if d.startswith(("GLIDE_ERR_", "GLIDE_TUNE_", "GLIDE_GROUP_TUNE_",
                                                "GLIDE_ENTH_TUNE_", "GLIDE_VTI_"))]
    assert len(must) >= 20
    checked = 0
    for d, v in defines.items():
        if d.startswith(("GLIDE_RESTRICT_", "GLIDE_PROLONG_")):
            op = d[len("GLIDE_"):].lower().replace("prolong_", "prolongate_")
            assert _lib.TRANSFER_OPS[op] == v, d
            checked += 1
            continue
        mirror = getattr(_lib, python_name(d), None)
        if mirror is None:
            assert d not in must, f"{d} has no Python mirror"
            continue
        assert mirror == v, (d, mirror, v)
        checked += 1
    assert checked >= 50


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "glide_forward" in names and "glide_enthalpy_column_sweep" in names
    assert len(names) >= 40


def test_library_exports_every_declared_symbol():
    from glide_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built")
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_table_covers_every_declared_symbol():
    from glide_b200 import _lib
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, missing
    if _lib.LIB_PATH.exists():
        _lib.load()  # binds every signature; raises if a name is absent


def test_version_and_error_text_without_gpu():
    from glide_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built")
    lib = _lib.load()
    assert lib.glide_version() >= 1
    # argument errors are reported before any device work
    h = ctypes.c_void_p()
    assert lib.glide_enthalpy_create(4, 4, 1, 1000.0, ctypes.byref(h)) == _lib.GLIDE_ERR_SHAPE
    assert b"nz" in lib.glide_enthalpy_last_error()
    assert lib.glide_create(0, 8, 1000.0, 1, 0, ctypes.byref(h)) != _lib.GLIDE_OK
