"""ctypes wrappers of the enthalpy restatement in enthalpy_oracle.cpp (test
infrastructure only).  Arrays use the reference's layouts: E-like arrays
(ny, nx, nz), u3d (nz, ny, nx+1), v3d (nz, ny+1, nx), 2-D arrays (ny, nx);
all binary64 and C-contiguous."""
from __future__ import annotations

import ctypes

import numpy as np

from .glide_oracle import lib

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int


def _p(a):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("arrays must be C-contiguous float64")
    return _P(a.ctypes.data)


def _declare():
    L = lib()
    if getattr(L, "_eo_declared", False):
        return L
    arr10 = [_P] * 10
    L.eo_residual.argtypes = arr10 + [_D] * 5 + [_I, _I, _I, _I, _I]
    L.eo_column_smooth.argtypes = arr10 + [_D] * 5 + [_I, _I, _I, _I, _I, _D]
    L.eo_layer_smooth.argtypes = arr10 + [_D] * 5 + [_I, _I, _I, _I]
    L.eo_compute_omega.argtypes = [_P] * 6 + [_D, _I, _I, _I]
    L.eo_e_scale.restype = _D
    L._eo_declared = True
    return L


def _common(s, cfg):
    return ([_p(s[k]) for k in ("E", "E_prev", "f_E", "u3d", "v3d", "omega", "H", "H_prev", "E_surface")],
            [cfg["dx"], cfg["dt"], cfg["drain_rate"], cfg["h_thin"], cfg["lf_c"], int(cfg["term_flags"])])


def residual(s: dict, cfg: dict, use_forcing: bool = True) -> np.ndarray:
    L = _declare()
    ny, nx, nz = s["E"].shape
    out = np.zeros_like(s["E"])
    arrs, sc = _common(s, cfg)
    L.eo_residual(_p(out), *arrs, *sc, int(use_forcing), ny, nx, nz)
    return out


def column_smooth(s: dict, cfg: dict) -> np.ndarray:
    L = _declare()
    ny, nx, nz = s["E"].shape
    out = np.zeros_like(s["E"])
    arrs, sc = _common(s, cfg)
    L.eo_column_smooth(_p(out), *arrs, *sc, ny, nx, nz, int(cfg["n_newton"]), float(cfg["relaxation"]))
    return out


def layer_smooth(s: dict, cfg: dict) -> np.ndarray:
    L = _declare()
    ny, nx, nz = s["E"].shape
    out = np.zeros_like(s["E"])
    arrs, sc = _common(s, cfg)
    L.eo_layer_smooth(_p(out), *arrs, *sc, ny, nx, nz)
    return out


def compute_omega(u3d, v3d, H, dh_dt, bmb, dx) -> np.ndarray:
    L = _declare()
    ny, nx = H.shape
    nz = u3d.shape[0]
    out = np.zeros((ny, nx, nz))
    L.eo_compute_omega(_p(out), _p(u3d), _p(v3d), _p(H), _p(dh_dt), _p(bmb), float(dx), ny, nx, nz)
    return out


def column_sweep(s: dict, cfg: dict, n_iter: int, alternating: bool = True):
    """EnthalpyOperators.column_sweep (glide/enthalpy.py:426-471) on s["E"]
    in place; returns the residual max-norms [r0, r1, ...]."""
    r0 = float(np.max(np.abs(residual(s, cfg))))
    norms = [r0]
    for _ in range(n_iter):
        s["E"] += cfg["omega"] * column_smooth(s, cfg)
        if alternating:
            s["E"] += cfg["omega"] * layer_smooth(s, cfg)
        r = float(np.max(np.abs(residual(s, cfg))))
        norms.append(r)
        rel = r / r0 if r0 > 0 else 0.0
        if rel < cfg["relative_tolerance"] or r < cfg["absolute_tolerance"]:
            break
    return norms


SEC_PER_YR = 365.25 * 86400.0
E_SCALE_HOST = 2009.0 * (273.15 - 223.15)


def temperature(E, H, nz):
    """EnthalpyOperators.get_temperature (glide/enthalpy.py:565-581)."""
    sigma = np.linspace(0.0, 1.0, nz)
    T = np.zeros_like(E)
    for k in range(nz):
        depth = (1.0 - float(sigma[k])) * H
        T_pmp = 273.15 - 7.9e-8 * 910.0 * 9.81 * depth
        T[:, :, k] = np.minimum(E[:, :, k] * E_SCALE_HOST / 2009.0 + 223.15, T_pmp)
    return T


def arrhenius_B(E, H, nz, n_glen=3.0):
    """EnthalpyOperators.get_arrhenius_factor (glide/enthalpy.py:600-643)."""
    sigma = np.linspace(0.0, 1.0, nz)
    T = temperature(E, H, nz)
    A = np.where(T < 263.15, 3.985e-13, 1.916e3) * np.exp(-np.where(T < 263.15, 60e3, 139e3)
                                                         / (8.314 * np.maximum(T, 1.0)))
    for k in range(nz):
        depth = (1.0 - float(sigma[k])) * H
        T_pmp = 273.15 - 7.9e-8 * 910.0 * 9.81 * depth
        w = np.maximum(E[:, :, k] * E_SCALE_HOST - 2009.0 * (T_pmp - 223.15), 0.0) / 334000.0
        A[:, :, k] *= (1.0 + 181.25 * w)
    return np.mean(A, axis=2) ** (-1.0 / n_glen)


def _cfg(dx, dt):
    """EnthalpyOperators' default term and smoother settings
    (glide/enthalpy.py:205-300)."""
    return dict(dx=dx, dt=dt, drain_rate=0.01 / SEC_PER_YR, h_thin=25.0, lf_c=1e-12, term_flags=7, omega=1.0,
                n_newton=3, relaxation=1.0, relative_tolerance=1e-5, absolute_tolerance=1e-2)


class OracleThermal:
    """ThermalModel (glide/model.py:97-222) over the restated kernels, with
    state kept between steps: initialize, pre_momentum, step."""

    def __init__(self, dx, nz, n_smooth=10, m=1.0, u_reg=1.0, rho_i=917.0, n_glen=3.0):
        self.dx, self.nz, self.n_smooth = dx, nz, n_smooth
        self.m, self.u_reg, self.rho_i, self.n_glen = m, u_reg, rho_i, n_glen
        self.sigma = np.linspace(0.0, 1.0, nz)

    def set_surface_temperature(self, T_s):
        """set_surface_enthalpy_from_temperature (glide/enthalpy.py:521-530)."""
        self.E_s = 2009.0 * (np.minimum(T_s, 273.15) - 223.15) / E_SCALE_HOST

    def initialize(self, T_s, H, Q_geo):
        """ThermalModel.initialize (glide/model.py:134-153) with T_field =
        T_surface, capped at the pressure-melting point of each level."""
        ny, nx = H.shape
        T = np.broadcast_to(T_s[:, :, None], (ny, nx, self.nz)).copy()
        for k in range(self.nz):
            T_pmp = 273.15 - 7.9e-8 * 910.0 * 9.81 * ((1.0 - float(self.sigma[k])) * H)
            T[:, :, k] = np.minimum(T[:, :, k], T_pmp)
        self.E = 2009.0 * (T - 223.15) / E_SCALE_HOST
        self.E_prev, self.H_prev = self.E.copy(), H.copy()
        self.set_surface_temperature(T_s)
        self.Q_geo = Q_geo

    def pre_momentum(self, H):
        """glide/model.py:155-164."""
        self.E_prev = self.E.copy()
        self.H_prev = H.copy()

    def step(self, u, v, H1, beta, dt):
        """ThermalModel.step (glide/model.py:166-222): omega from the realised
        thickness change in m/a, the velocity in m/s, frictional heating,
        forcing, column sweeps; returns B in the momentum solver's units."""
        ny, nx = H1.shape
        nz = self.nz
        u3 = np.ascontiguousarray(np.broadcast_to(u, (nz,) + u.shape))
        v3 = np.ascontiguousarray(np.broadcast_to(v, (nz,) + v.shape))
        dt_yr = dt / SEC_PER_YR
        omega = compute_omega(u3, v3, H1, (H1 - self.H_prev) / dt_yr, np.zeros((ny, nx)), self.dx) / SEC_PER_YR
        u3 = u3 / SEC_PER_YR
        v3 = v3 / SEC_PER_YR
        uc = 0.5 * (u3[0][:, 1:] + u3[0][:, :-1])
        vc = 0.5 * (v3[0][1:, :] + v3[0][:-1, :])
        self.Q_fh = beta * np.sqrt(uc ** 2 + vc ** 2 + self.u_reg ** 2) ** (self.m + 1.0)
        dsig_half = 0.5 * (1.0 / (nz - 1))
        f_E = np.zeros((ny, nx, nz))
        f_E[:, :, 0] += (self.Q_geo + self.Q_fh) / (dsig_half * E_SCALE_HOST)
        st = dict(E=self.E, E_prev=self.E_prev, f_E=f_E, u3d=u3, v3d=v3, omega=np.ascontiguousarray(omega), H=H1,
                  H_prev=self.H_prev, E_surface=self.E_s)
        self.sweep_norms = column_sweep(st, _cfg(self.dx, dt), self.n_smooth)
        self.E = st["E"]
        self.omega = omega
        return arrhenius_B(self.E, H1, nz, self.n_glen) / (self.rho_i * 9.81 * SEC_PER_YR ** (1.0 / self.n_glen))


def thermal_step(u, v, H0, H1, beta, T_s, Q_geo, dx, nz, n_smooth, dt, m=1.0, u_reg=1.0, rho_i=917.0,
                 n_glen=3.0):
    """ThermalModel initialize -> pre_momentum -> (H0 becomes H1) -> step(dt)
    (glide/model.py:134-222), with the restated kernels; returns E, omega,
    Q_fh, B, T in the reference's layouts."""
    tm = OracleThermal(dx, nz, n_smooth, m=m, u_reg=u_reg, rho_i=rho_i, n_glen=n_glen)
    tm.initialize(T_s, H0, Q_geo)
    tm.pre_momentum(H0)
    B = tm.step(u, v, H1, beta, dt)
    return dict(E=tm.E, omega=tm.omega, Q_fh=tm.Q_fh, B=B, T=temperature(tm.E, H1, nz))
