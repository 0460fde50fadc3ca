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
