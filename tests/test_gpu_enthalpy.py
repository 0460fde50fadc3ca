"""GPU tests of the enthalpy column solver (include/glide_enthalpy.h) through
the EnthalpyOperators / ThermalModel mirror: against the reference's own
outputs (golden fixtures), against the oracle on larger seeded states, and
against the analytic answers of the reference's enthalpy tests.

Tolerances (binary64): single operators 1e-12 relative to the largest
entry; column Newton/Thomas results and sweeps 1e-10; a full thermal step
1e-10."""
from __future__ import annotations

import numpy as np
import pytest

from cases import SEC_PER_YR, enthalpy_config, enthalpy_state
from util import load_golden, rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _ops(st, dx, nz):
    from glide_b200.enthalpy import EnthalpyOperators
    from glide_b200.grid import Grid
    ny, nx = st["H"].shape
    g = Grid(ny, nx, dx)
    g.state.H.set(torch.as_tensor(st["H"]))
    ops = EnthalpyOperators(g, nz=nz)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    ops.enthalpy_state.E[:] = T(st["E"])
    ops.enthalpy_state.E_prev[:] = T(st["E_prev"])
    ops.f_E[:] = T(st["f_E"])
    ops.enthalpy_velocity.u3d[:] = T(st["u3d"])
    ops.enthalpy_velocity.v3d[:] = T(st["v3d"])
    ops.enthalpy_velocity.omega[:] = T(st["omega"])
    ops.H_prev[:] = T(st["H_prev"])
    ops.enthalpy_forcing.E_surface[:] = T(st["E_surface"])
    return ops


def _golden_state(g):
    return {k: g[f"in_{k}"] for k in ("E", "E_prev", "f_E", "u3d", "v3d", "omega", "H", "H_prev", "E_surface")}


def test_operators_match_reference():
    g = load_golden("enthalpy_ops_f64")
    cfg = enthalpy_config()
    ops = _ops(_golden_state(g), cfg["dx"], g["in_E"].shape[2])
    dt = cfg["dt"]
    rmax = ops.compute_residual(dt)
    assert rel_err(_np(ops.r_E), g["out_r_E"]) <= 1e-12
    assert abs(rmax - float(g["out_rmax"])) <= 1e-12 * float(g["out_rmax"])
    ops.column_smooth(dt)
    assert rel_err(_np(ops.delta_E), g["out_column_delta"]) <= 1e-10
    ops.layer_smooth(dt)
    assert rel_err(_np(ops.delta_E), g["out_layer_delta"]) <= 1e-12
    ops.enthalpy_velocity.u3d[:] = torch.as_tensor(g["in_u3d"] * SEC_PER_YR, device="cuda")
    ops.enthalpy_velocity.v3d[:] = torch.as_tensor(g["in_v3d"] * SEC_PER_YR, device="cuda")
    ops.compute_omega(torch.as_tensor(g["in_dh_dt"], device="cuda"))
    assert rel_err(_np(ops.enthalpy_velocity.omega), g["out_omega"]) <= 1e-12


@pytest.mark.parametrize("tag,alternating,n", [("alt", True, 4), ("col", False, 3)])
def test_column_sweep_matches_reference(tag, alternating, n):
    g = load_golden("enthalpy_ops_f64")
    cfg = enthalpy_config()
    ops = _ops(_golden_state(g), cfg["dx"], g["in_E"].shape[2])
    ops.smoother_config.relative_tolerance = 1e-30
    ops.smoother_config.absolute_tolerance = 0.0
    ops.column_sweep(cfg["dt"], n, alternating=alternating)
    assert ops.last_stats.iterations == n
    assert rel_err(_np(ops.enthalpy_state.E), g[f"out_sweep_{tag}_E"]) <= 1e-10


def test_column_sweep_stop_test_matches_oracle():
    """The device-side stop test takes the same number of sweeps as the
    reference's host loop (glide/enthalpy.py:457-471)."""
    from oracle import enthalpy_oracle as eo
    st = enthalpy_state(20, 24, 17, seed=9)
    cfg = enthalpy_config(relative_tolerance=1e-3)
    s = {k: v.copy() for k, v in st.items()}
    norms = eo.column_sweep(s, cfg, 30)
    ops = _ops(st, cfg["dx"], 17)
    ops.smoother_config.relative_tolerance = 1e-3
    ops.column_sweep(cfg["dt"], 30)
    assert ops.last_stats.iterations == len(norms) - 1
    assert rel_err(_np(ops.enthalpy_state.E), s["E"]) <= 1e-10


def test_larger_state_matches_oracle():
    from oracle import enthalpy_oracle as eo
    st = enthalpy_state(48, 64, 41, seed=11)
    cfg = enthalpy_config(relative_tolerance=1e-30, absolute_tolerance=0.0)
    ops = _ops(st, cfg["dx"], 41)
    ops.smoother_config.relative_tolerance = 1e-30
    ops.smoother_config.absolute_tolerance = 0.0
    s = {k: v.copy() for k, v in st.items()}
    ops.compute_residual(cfg["dt"])
    assert rel_err(_np(ops.r_E), eo.residual(s, cfg)) <= 1e-12
    eo.column_sweep(s, cfg, 3)
    ops.column_sweep(cfg["dt"], 3)
    assert rel_err(_np(ops.enthalpy_state.E), s["E"]) <= 1e-10


def test_thermal_step_matches_reference():
    from glide_b200.grid import Grid
    from glide_b200.model import ThermalModel
    g = load_golden("thermal_step_f64")
    ny, nx = g["in_H0"].shape
    nz = g["out_E"].shape[2]
    grid = Grid(ny, nx, 1500.0)
    T = lambda a: torch.as_tensor(a)
    grid.state.u.set(T(g["in_u"]))
    grid.state.v.set(T(g["in_v"]))
    grid.state.H.set(T(g["in_H0"]))
    grid.sliding.beta.set(T(g["in_beta"]))
    tm = ThermalModel(grid, nz=nz, n_smooth=4)
    tm.initialize(T(g["in_T_s"]), Q_geo=0.05)
    tm.pre_momentum()
    grid.state.H.set(T(g["in_H1"]))
    tm.step(float(g["in_dt"]))
    assert rel_err(_np(tm.enthalpy), g["out_E"]) <= 1e-10
    assert rel_err(_np(tm.ops.enthalpy_velocity.omega), g["out_omega"]) <= 1e-10
    assert rel_err(_np(tm.ops.enthalpy_forcing.Q_fh), g["out_Q_fh"]) <= 1e-12
    assert rel_err(_np(grid.rheology.B.data), g["out_B"]) <= 1e-10
    assert rel_err(_np(tm.temperature), g["out_T"]) <= 1e-10


def test_cold_column_analytic():
    """tests/test_enthalpy_cold_column.py of the reference: steady cold column
    within 5e-3 of E(sigma) = E_s + c_i Q_geo H / k_i (1 - sigma)."""
    from glide_b200.enthalpy import C_I, E_SCALE, K_I, T_REF, EnthalpyOperators
    from glide_b200.grid import Grid
    ny = nx = 4
    nz, H, Ts, Q = 21, 1000.0, 243.15, 0.04
    g = Grid(ny, nx, 1000.0)
    g.state.H.set(torch.full((ny, nx), H, dtype=torch.float64))
    ops = EnthalpyOperators(g, nz=nz)
    ops.term_flags.horizontal_advection = False
    ops.initialize_from_temperature(Ts)
    ops.set_surface_enthalpy_from_temperature(torch.full((ny, nx), Ts, dtype=torch.float64))
    ops.enthalpy_forcing.Q_geo[:, :] = Q
    dt = 1000.0 * SEC_PER_YR
    for _ in range(200):
        ops.set_rhs()
        ops.column_sweep(dt, 20)
    sigma = np.linspace(0.0, 1.0, nz)
    E = _np(ops.enthalpy_state.E[ny // 2, nx // 2, :]) * E_SCALE
    Ea = C_I * (Ts - T_REF) + C_I * Q * H / K_I * (1 - sigma)
    assert np.max(np.abs(E[:-1] - Ea[:-1]) / np.abs(Ea[:-1])) < 5e-3


@pytest.mark.parametrize("nz", [3, 4, 17])
def test_column_sweeps_match_oracle_across_nz(nz):
    """A 3-sweep column solve at the smallest column heights and an odd one
    (thin-ice columns included) against the oracle at 1e-10."""
    from oracle import enthalpy_oracle as eo
    st = enthalpy_state(24, 40, nz, seed=13)
    cfg = enthalpy_config(relative_tolerance=1e-30, absolute_tolerance=0.0)
    ops = _ops(st, cfg["dx"], nz)
    ops.smoother_config.relative_tolerance = 1e-30
    ops.smoother_config.absolute_tolerance = 0.0
    ops.column_sweep(cfg["dt"], 3)
    s = {k: v.copy() for k, v in st.items()}
    eo.column_sweep(s, cfg, 3)
    assert rel_err(_np(ops.enthalpy_state.E), s["E"]) <= 1e-10


@pytest.mark.parametrize("nz", [3, 4, 17, 41])
@pytest.mark.parametrize("flat", [True, False])
def test_column_kernels_agree_and_match_oracle(nz, flat):
    """The column smoother with its factors in shared memory (the default)
    against the one-thread-per-column kernel (1e-12) and, over three
    alternating sweeps, against the oracle (1e-10).  flat: one velocity for
    every layer, read in place from the grid (the coupled model's case,
    where the horizontal flux of the frozen neighbours is folded into the
    row constants); otherwise a velocity per layer."""
    from oracle import enthalpy_oracle as eo
    st = enthalpy_state(40, 52, nz, seed=nz)
    if flat:
        st["u3d"] = np.ascontiguousarray(np.broadcast_to(st["u3d"][0], st["u3d"].shape))
        st["v3d"] = np.ascontiguousarray(np.broadcast_to(st["v3d"][0], st["v3d"].shape))
    cfg = enthalpy_config(relative_tolerance=1e-30, absolute_tolerance=0.0)
    out = {}
    for kernel in ("local", "smem8", "smem"):
        ops = _ops(st, cfg["dx"], nz)
        if flat:
            ops.grid.state.u.set(torch.as_tensor(st["u3d"][0]))
            ops.grid.state.v.set(torch.as_tensor(st["v3d"][0]))
            ops.broadcast_velocity()
        ops.set_tuning(column_kernel=kernel)
        ops.column_smooth(cfg["dt"])
        out[kernel] = _np(ops.delta_E).copy()
        if kernel == "smem":
            ops.smoother_config.relative_tolerance = 1e-30
            ops.smoother_config.absolute_tolerance = 0.0
            ops.column_sweep(cfg["dt"], 3)
            s = {k: v.copy() for k, v in st.items()}
            eo.column_sweep(s, cfg, 3)
            assert rel_err(_np(ops.enthalpy_state.E), s["E"]) <= 1e-10
    assert rel_err(out["smem"], out["local"]) <= 1e-12
    assert rel_err(out["smem8"], out["smem"]) <= 1e-15
