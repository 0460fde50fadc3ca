"""Coupled thermomechanical time steps on the oracle (test infrastructure only).

Restates the step loop of the reference's coupled example
(examples/thermal/coupled_dome.py:258-272) over the restated kernels:

    ThermalModel.pre_momentum()          E_prev <- E, H_prev <- H  (glide/model.py:155-164)
    IceDynamics.forward(t, dt_yr)        FASCD solve, then H_prev <- H on the top level
                                         (glide/model.py:65-72)
    set_surface_enthalpy_from_temperature(T_s(H, bed))
    ThermalModel.step(dt_s)              omega, frictional heating, forcing, column
                                         sweeps, B fed back into the top level only
                                         (glide/model.py:166-222); in native mode
                                         (quirks=False) restricted to every level

The surface temperature is the large-run recipe's lapse law,
T_s = 273.15 + (-30 + 6e-3 (2000 - s)) K with s = max(bed + H, (1 - 0.917) H).
"""
from __future__ import annotations

import numpy as np

from .enthalpy_oracle import SEC_PER_YR, OracleThermal, arrhenius_B
from .glide_oracle import OracleHierarchy


def surface_temperature(H, bed):
    s = np.maximum(bed + H, (1.0 - 0.917) * H)
    return 273.15 + (-30.0 + 6e-3 * (2000.0 - s))


def coupled_run(f, dx, n_levels, nz, dt_yr, n_steps, vcycles, Q_geo=0.05, n_smooth=10, quirks=True,
                init_B=True):
    """n_steps coupled steps from the fields f (bed, B, beta, smb, H, H_prev),
    each SSA solve exactly `vcycles` FASCD V-cycles (no tolerance test);
    returns the level-0 u, v, H, the enthalpy E (ny, nx, nz), the fed-back B
    and the column-sweep residual norms of each step."""
    ny, nx = f["H"].shape
    o = OracleHierarchy(ny, nx, dx, n_levels, reference_quirks=quirks)
    for k in ("bed", "B", "beta", "smb", "H", "H_prev"):
        o.set_field(k, f[k])
    o.fas.maximum_vcycles, o.fas.relative_tolerance, o.fas.absolute_tolerance = vcycles, 0.0, 0.0
    top = o.levels[0]
    tm = OracleThermal(dx, nz, n_smooth)
    tm.initialize(surface_temperature(top.H, top.bed), top.H.copy(), Q_geo)
    if init_B:  # the reference example's start (coupled_dome.py:144-146): B set on every level
        o.set_field("B", arrhenius_B(tm.E, top.H, nz) / (tm.rho_i * 9.81 * SEC_PER_YR ** (1.0 / tm.n_glen)))
    dt_s = dt_yr * SEC_PER_YR
    sweeps = []
    for _ in range(n_steps):
        tm.pre_momentum(top.H)
        o.solve(dt_yr)
        top.H_prev[...] = top.H
        tm.set_surface_temperature(surface_temperature(top.H, top.bed))
        top.B[...] = tm.step(top.u, top.v, top.H.copy(), top.beta, dt_s)
        if not quirks:  # native mode restricts the fed-back B to every level
            o.set_field("B", top.B.copy())
        sweeps.append(len(tm.sweep_norms) - 1)
    return dict(u=top.u.copy(), v=top.v.copy(), H=top.H.copy(), E=tm.E.copy(), B=top.B.copy(), sweeps=sweeps)
