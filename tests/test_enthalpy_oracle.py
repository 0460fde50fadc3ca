"""The enthalpy restatement (oracle/enthalpy_oracle.cpp) against the
reference's own enthalpy kernels and Python (golden fixtures made by
tests/golden/make_golden.py) and against the analytic answers of the
reference's enthalpy tests (tests/test_enthalpy_cold_column.py,
tests/test_enthalpy_stefan.py)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from cases import SEC_PER_YR, enthalpy_config
from util import load_golden, rel_err

eo = pytest.importorskip("oracle.enthalpy_oracle")


def _state(g):
    return {k: np.ascontiguousarray(g[f"in_{k}"]) for k in
            ("E", "E_prev", "f_E", "u3d", "v3d", "omega", "H", "H_prev", "E_surface")}


def test_operators_match_reference():
    g = load_golden("enthalpy_ops_f64")
    s, cfg = _state(g), enthalpy_config()
    assert rel_err(eo.residual(s, cfg), g["out_r_E"]) <= 1e-12
    assert rel_err(eo.column_smooth(s, cfg), g["out_column_delta"]) <= 1e-12
    assert rel_err(eo.layer_smooth(s, cfg), g["out_layer_delta"]) <= 1e-12
    om = eo.compute_omega(s["u3d"] * SEC_PER_YR, s["v3d"] * SEC_PER_YR, s["H"], g["in_dh_dt"],
                          np.zeros_like(s["H"]), cfg["dx"])
    assert rel_err(om, g["out_omega"]) <= 1e-12


@pytest.mark.parametrize("tag,alternating,n", [("alt", True, 4), ("col", False, 3)])
def test_column_sweep_matches_reference(tag, alternating, n):
    g = load_golden("enthalpy_ops_f64")
    s = _state(g)
    cfg = enthalpy_config(relative_tolerance=1e-30, absolute_tolerance=0.0)
    eo.column_sweep(s, cfg, n, alternating=alternating)
    assert rel_err(s["E"], g[f"out_sweep_{tag}_E"]) <= 1e-10


def test_thermal_step_matches_reference():
    g = load_golden("thermal_step_f64")
    nz = g["out_E"].shape[2]
    got = eo.thermal_step(g["in_u"], g["in_v"], g["in_H0"], g["in_H1"], g["in_beta"], g["in_T_s"], 0.05, 1500.0,
                          nz, 4, float(g["in_dt"]))
    for k in ("E", "omega", "Q_fh", "B", "T"):
        assert rel_err(got[k], g[f"out_{k}"]) <= 1e-10, k


def _cold_column(nz=21, H=1000.0, Ts=243.15, Q=0.04):
    ny = nx = 4
    sig = np.linspace(0.0, 1.0, nz)
    E0 = 2009.0 * (Ts - 223.15) / eo.E_SCALE_HOST
    z = np.zeros((ny, nx, nz))
    s = dict(E=z + E0, E_prev=z + E0, f_E=z.copy(), u3d=np.zeros((nz, ny, nx + 1)), v3d=np.zeros((nz, ny + 1, nx)),
             omega=z.copy(), H=np.full((ny, nx), H), H_prev=np.full((ny, nx), H), E_surface=np.full((ny, nx), E0))
    return s, sig, E0


def test_cold_column_analytic():
    """Steady cold column: E(sigma) = E_s + c_i Q_geo H / k_i (1 - sigma)
    within 5e-3 (the tolerance of tests/test_enthalpy_cold_column.py:128)."""
    s, sig, E0 = _cold_column()
    nz = len(sig)
    cfg = enthalpy_config(dt=1000.0 * SEC_PER_YR, term_flags=2 | 4)
    dsig_half = 0.5 / (nz - 1)
    for _ in range(60):
        s["E_prev"] = s["E"].copy()
        s["f_E"] = np.zeros_like(s["E"])
        s["f_E"][:, :, 0] = 0.04 / (dsig_half * eo.E_SCALE_HOST)
        eo.column_sweep(s, cfg, 20)
    E = s["E"][2, 2] * eo.E_SCALE_HOST
    Ea = E0 * eo.E_SCALE_HOST + 2009.0 * 0.04 * 1000.0 / 2.1 * (1 - sig)
    assert np.max(np.abs(E[:-1] - Ea[:-1]) / np.abs(Ea[:-1])) < 5e-3


def test_cold_column_smoother_reduces_residual():
    """tests/test_enthalpy_cold_column.py:137-192: 50 column smooths cut the
    residual more than 100-fold."""
    s, sig, E0 = _cold_column()
    nz = len(sig)
    cfg = enthalpy_config(dt=1000.0 * SEC_PER_YR, term_flags=2 | 4)
    s["f_E"][:, :, 0] = 0.04 / (0.5 / (nz - 1) * eo.E_SCALE_HOST)
    r = []
    for _ in range(50):
        r.append(np.max(np.abs(eo.residual(s, cfg))))
        s["E"] += eo.column_smooth(s, cfg)
    assert r[0] / r[-1] > 100


REF = os.environ.get("GLIDE_REFERENCE", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "glide", "cuda")),
                    reason="reference checkout not present")
@pytest.mark.parametrize("nz,flags", [(3, 7), (4, 1), (17, 6), (24, 0), (41, 7)])
def test_oracle_matches_live_reference_across_nz_and_terms(nz, flags):
    """Fresh states of several column heights and term selections (bit 1
    horizontal advection, 2 sigma advection, 4 drainage), the reference's
    EnthalpyOperators run live (its kernels on host cores): residual, column
    and layer smoothers at 1e-12, and a 3-sweep alternating solve at 1e-10."""
    import contextlib
    import io

    from cases import enthalpy_state
    from oracle import build_oracle
    from oracle.refpy import load_reference
    build_oracle.build_reference(REF)
    load_reference(fp64=True, reference=REF)
    from glide.enthalpy import EnthalpyOperators, EnthalpyTermFlags
    from glide.grid import Grid
    ny, nx = 5, 7
    st = enthalpy_state(ny, nx, nz, seed=31 + nz)
    cfg = enthalpy_config(term_flags=flags, relative_tolerance=1e-30, absolute_tolerance=0.0)
    dt = cfg["dt"]

    def make_ops():
        with contextlib.redirect_stdout(io.StringIO()):
            g = Grid(ny, nx, cfg["dx"])
            g.state.H.set(st["H"])
            ops = EnthalpyOperators(g, nz=nz)
        ops.term_flags = EnthalpyTermFlags(horizontal_advection=bool(flags & 1), omega=bool(flags & 2),
                                           drainage=bool(flags & 4))
        es, ev, ef = ops.enthalpy_state, ops.enthalpy_velocity, ops.enthalpy_forcing
        es.E[:] = st["E"]
        es.E_prev[:] = st["E_prev"]
        ops.f_E[:] = st["f_E"]
        ev.u3d[:] = st["u3d"]
        ev.v3d[:] = st["v3d"]
        ev.omega[:] = st["omega"]
        ops.H_prev[:] = st["H_prev"]
        ef.E_surface[:] = st["E_surface"]
        ops.smoother_config.relative_tolerance = 1e-30
        ops.smoother_config.absolute_tolerance = 0.0
        return ops

    s = {k: np.ascontiguousarray(v.copy()) for k, v in st.items()}
    ops = make_ops()
    with contextlib.redirect_stdout(io.StringIO()):
        ops.compute_residual(dt)
    assert rel_err(eo.residual(s, cfg), np.array(ops.r_E)) <= 1e-12
    with contextlib.redirect_stdout(io.StringIO()):
        ops.column_smooth(dt)
    assert rel_err(eo.column_smooth(s, cfg), np.array(ops.delta_E)) <= 1e-12
    with contextlib.redirect_stdout(io.StringIO()):
        ops.layer_smooth(dt)
    assert rel_err(eo.layer_smooth(s, cfg), np.array(ops.delta_E)) <= 1e-12
    ops = make_ops()
    with contextlib.redirect_stdout(io.StringIO()):
        ops.column_sweep(dt, 3, alternating=True)
    eo.column_sweep(s, cfg, 3, alternating=True)
    assert rel_err(s["E"], np.array(ops.enthalpy_state.E)) <= 1e-10
