"""Shared helpers of the test suite: fixture loading, oracle set-up and the
relative-difference measure the parity tests use."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_golden(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def rel_err(a, b):
    """max |a - b| / max(max |b|, tiny): a scale-aware max-norm difference."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def oracle_single_level(inp, dx, dtype=np.float64, calving=0.0):
    """One-level oracle hierarchy loaded with a random-state fixture."""
    from oracle.glide_oracle import OracleHierarchy
    ny, nx = inp["in_H"].shape
    o = OracleHierarchy(ny, nx, dx, 1, dtype=dtype)
    for k in ("u", "v", "H", "H_prev", "mask", "bed", "B", "beta", "smb"):
        o.set_field(k, inp[f"in_{k}"])
    lev = o.levels[0]
    lev.f_u[...] = inp["in_f_u"]
    lev.f_v[...] = inp["in_f_v"]
    o.set_phys(calving_rate=calving)
    return o


def oracle_c1(inp, n_levels=4, dx=1000.0, dtype=np.float64):
    from oracle.glide_oracle import OracleHierarchy
    ny, nx = inp["in_H"].shape
    o = OracleHierarchy(ny, nx, dx, n_levels, dtype=dtype)
    for k in ("bed", "B", "beta", "smb", "H", "H_prev"):
        o.set_field(k, inp[f"in_{k}"])
    return o
