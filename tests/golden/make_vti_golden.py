"""Generate the VTI/PVD golden files in tests/golden/vti/ with the reference's
own writer (glide/io.py write_vti and VTIWriter of JacobDowns/glide).

The reference package is imported on host cores through oracle/refpy.py's
CuPy stand-in (cupy.asnumpy is numpy.asarray there; the writer itself is
pure NumPy and xml.etree).  Face fields are the reference's own Field objects,
so their to_cell averaging is the reference's.  Inputs are stored beside the
files in vti/inputs.npz.

    python tests/golden/make_vti_golden.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import importlib
import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle.refpy import DEFAULT_REFERENCE, load_reference  # noqa: E402

OUT = HERE / "vti"


def inputs():
    rng = np.random.default_rng(2024)
    ny, nx, nz = 6, 5, 3
    f = {
        "H": rng.uniform(0.0, 3000.0, (ny, nx)).astype(np.float32),
        "u": rng.normal(0.0, 50.0, (ny, nx + 1)).astype(np.float32),
        "v": rng.normal(0.0, 50.0, (ny + 1, nx)),  # binary64: to_cell in binary64, then rounded
        "B": rng.uniform(1e7, 2e8, (ny, nx)),
        "bed": rng.normal(0.0, 400.0, (ny, nx)).astype(np.float32),
        "a": rng.normal(size=(ny, nx)),
        "b": rng.normal(size=(ny, nx)).astype(np.float32),
        "c": rng.normal(size=(ny, nx)),
        "E": rng.normal(size=(ny, nx, nz)),
        "T": rng.normal(260.0, 5.0, (ny, nx, nz)).astype(np.float32),
        "H1": rng.uniform(0.0, 3000.0, (ny, nx)).astype(np.float32),
    }
    return f


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    a = ap.parse_args()
    load_reference(fp64=False, reference=a.reference)
    rio = importlib.import_module("glide.io")
    rfield = importlib.import_module("glide.field")
    Field, GE = rfield.Field, rfield.GridEntity
    f = inputs()
    if OUT.exists():
        shutil.rmtree(OUT)
    OUT.mkdir(parents=True)
    np.savez(OUT / "inputs.npz", **f)
    u = Field(data=f["u"], grid_entity=GE.VERTICAL_FACET, dx=1000.0)
    v = Field(data=f["v"], grid_entity=GE.HORIZONTAL_FACET, dx=1000.0)
    H = Field(data=f["H"], grid_entity=GE.CELL, dx=1000.0)

    # 2-D scalars and a 2-component vector of face fields, time value, flip
    rio.write_vti(OUT / "scalars_vector2.vti", {"H": H.data, "U": [u.to_cell().data, v.to_cell().data],
                                                "B": f["B"]},
                  1000.0, origin=(100.0, -50.0), time_value=2.5)
    # no flip, no time value, dy given, a 3-component vector (declared Vectors)
    rio.write_vti(OUT / "vector3_noflip.vti", {"W": [f["a"], f["b"], f["c"]], "bed": f["bed"]},
                  250.0, dy=500.0, flip_y=False)
    # 3-D scalars (ny, nx, nz), binary64 and binary32
    rio.write_vti(OUT / "volume.vti", {"E": f["E"], "T": f["T"]}, 2000.0, dz=0.5,
                  origin=(1.0, 2.0, 3.0), time_value=10)

    # VTIWriter: static + dynamic fields (Field objects, a vector of faces, a
    # callable), two snapshots and the PVD manifest
    state = {"H": f["H"]}
    w = rio.VTIWriter(out_dir=OUT / "series", base="dome", dx=1000.0, origin=(0.0, 0.0),
                      static_fields={"bed": f["bed"]},
                      dynamic_fields={"H": H, "U": [u, v], "Hsq": lambda: state["H"] * 2.0})
    w.initialize(None)
    w.append(None, time=0.0)
    H.data = f["H1"]
    state["H"] = f["H1"]
    w.append(None, time=5.0)
    w.write_pvd()
    for p in sorted(OUT.rglob("*")):
        if p.is_file():
            print(p.relative_to(OUT), p.stat().st_size)


if __name__ == "__main__":
    main()
