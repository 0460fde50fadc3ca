"""Enthalpy column solver (mirror of glide/enthalpy.py).

Same names and semantics as the reference's `EnthalpyOperators`:
compute_residual, column_smooth, layer_smooth, column_sweep, compute_omega,
set_rhs and the temperature conversions, over the C ABI of
include/glide_enthalpy.h (binary64 CUDA kernels).

Arrays keep the reference's shapes: E-like arrays (ny, nx, nz), u3d
(nz, ny, nx+1), v3d (nz, ny+1, nx).  On the device the 3-D node arrays are
layer-major, so the (ny, nx, nz) tensors here are strided views (strides
(nx, 1, ny*nx)) of that memory; in-place writes land in the solver's
arrays.  Internally E is scaled by E_SCALE, as in the reference.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Callable

import torch

from . import _lib
from ._lib import GlideError
from .field import Constant

# Physical constants (glide/enthalpy.py:46-65)
RHO_I = 910.0
RHO_W = 1000.0
C_I = 2009.0
K_I = 2.1
L_HEAT = 3.34e5
T_REF = 223.15
T_MELT = 273.15
BETA_CC = 7.9e-8
GRAVITY = 9.81
K_COLD = K_I / C_I
K_TEMP_FACTOR = 1e-1
K_TEMP = K_COLD * K_TEMP_FACTOR
E_SCALE = C_I * (T_MELT - T_REF)
SEC_PER_YR = 365.25 * 86400.0
MASS_FLUX_REG = 10.0 / (SEC_PER_YR ** 2)
MASS_FLUX_REG_YR = 10.0

FIELDS = ["E", "E_prev", "f_E", "omega", "r_E", "delta_E", "phi_strain", "u3d", "v3d", "H_prev",
          "E_surface", "Q_geo", "Q_fh"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}


def water_content_from_enthalpy(E, depth=0.0):
    """Water content from physical enthalpy (glide/enthalpy.py:68-72)."""
    T_pmp = T_MELT - BETA_CC * RHO_I * GRAVITY * depth
    E_pmp = C_I * (T_pmp - T_REF)
    return torch.clamp(E - E_pmp, min=0.0) / L_HEAT


def make_sigma(nz):
    """Uniform sigma levels from bed (0) to surface (1) (glide/enthalpy.py:75-93)."""
    return torch.linspace(0.0, 1.0, nz, dtype=torch.float64, device="cuda")


# ---------------------------------------------------------------- containers
@dataclass
class EnthalpyState:
    E: torch.Tensor | None = None
    E_prev: torch.Tensor | None = None

    def __repr__(self):
        return f"EnthalpyState: E {tuple(self.E.shape)}" if self.E is not None else "EnthalpyState: uninitialized"


@dataclass
class EnthalpyForcing:
    E_surface: torch.Tensor | None = None
    Q_geo: torch.Tensor | None = None
    Q_fh: torch.Tensor | None = None
    phi_strain: torch.Tensor | None = None
    drain_rate: Constant = field(default_factory=lambda: Constant(
        0.01 / (365.25 * 86400.0), name="drain_rate", units="s^{-1}",
        attrs={"long_name": "Water drainage rate in temperate ice (0.01 a^{-1} default)"}))
    h_thin: Constant = field(default_factory=lambda: Constant(
        25.0, name="h_thin", units="m",
        attrs={"long_name": "Thickness below which the column is clamped to the surface enthalpy (Dirichlet)"}))


class EnthalpyVelocity:
    """Layer velocities and omega.  `u3d` / `v3d` are the handle's own layer
    arrays; after `EnthalpyOperators.broadcast_velocity()` the kernels read
    the grid's 2-D velocity for every layer instead, and touching `u3d` or
    `v3d` copies that velocity into every layer first (what the reference's
    broadcast does eagerly)."""

    def __init__(self, ops):
        self._ops = ops

    @property
    def u3d(self):
        self._ops._materialize_velocity()
        return self._ops._view("u3d")

    @property
    def v3d(self):
        self._ops._materialize_velocity()
        return self._ops._view("v3d")

    @property
    def omega(self):
        return self._ops._view("omega")

    def __repr__(self):
        return f"EnthalpyVelocity: u3d {tuple(self.u3d.shape)}, v3d {tuple(self.v3d.shape)}"


@dataclass
class EnthalpyTermFlags:
    horizontal_advection: bool = True
    omega: bool = True
    drainage: bool = True

    @property
    def bitmask(self) -> int:
        return ((_lib.ENTH_HORIZ_ADV if self.horizontal_advection else 0)
                | (_lib.ENTH_SIGMA_DOT if self.omega else 0) | (_lib.ENTH_DRAINAGE if self.drainage else 0))


def _no_hook(i):
    return None


@dataclass
class ColumnSmootherConfig:
    omega: float = 1.0
    n_newton: int = 3
    relaxation: float = 1.0
    relative_tolerance: float = 1e-5
    absolute_tolerance: float = 1e-2
    lf_c: float = 1e-12
    report_norms: bool = False
    hook_func: Callable[[int], None] = field(default_factory=lambda: _no_hook)


class _Buf:
    def __init__(self, ptr, shape, strides, owner):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "strides": tuple(8 * s for s in strides),
                                         "typestr": "<f8", "data": (ptr, False), "version": 3}
        self._owner = owner


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ecall(name, *args):
    lib = _lib.load()
    code = getattr(lib, name)(*args)
    if code != _lib.GLIDE_OK:
        msg = lib.glide_enthalpy_last_error()
        raise GlideError(code, msg.decode() if msg else "")


class EnthalpyOperators:
    """Operators of the conservative enthalpy equation on one grid
    (glide/enthalpy.py:205-643); `grid` is a `glide_b200.grid.Grid` whose
    hierarchy is binary64 (or mixed).  `use_fast_math` is accepted for
    signature compatibility; the kernels here are binary64."""

    def __init__(self, grid, nz=11, use_fast_math=True):
        if grid._hier.dtype != torch.float64:
            raise NotImplementedError("the enthalpy solver runs in binary64: use a binary64 or mixed hierarchy")
        self.grid = grid
        self.nz = int(nz)
        self.sigma = make_sigma(self.nz)
        h = ctypes.c_void_p()
        _ecall("glide_enthalpy_create", int(grid.ny), int(grid.nx), self.nz, float(grid.dx), ctypes.byref(h))
        self._h = h
        self._views = {}
        self._broadcast = False
        self.enthalpy_state = _StateView(self)
        self.enthalpy_forcing = _ForcingView(self)
        self.enthalpy_velocity = EnthalpyVelocity(self)
        self.smoother_config = ColumnSmootherConfig()
        self.term_flags = EnthalpyTermFlags()
        self._vel_div = 1.0
        self._bind()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().glide_enthalpy_destroy(h)
            except Exception:
                pass
            self._h = None

    # -- memory ---------------------------------------------------------
    def _view(self, name):
        t = self._views.get(name)
        if t is not None:
            return t
        p = ctypes.c_void_p()
        _ecall("glide_enthalpy_field_ptr", self._h, FIELD_ID[name], ctypes.byref(p))
        ny, nx, nz = self.grid.ny, self.grid.nx, self.nz
        if name in ("u3d",):
            shape, strides = (nz, ny, nx + 1), (ny * (nx + 1), nx + 1, 1)
        elif name in ("v3d",):
            shape, strides = (nz, ny + 1, nx), ((ny + 1) * nx, nx, 1)
        elif name in ("H_prev", "E_surface", "Q_geo", "Q_fh"):
            shape, strides = (ny, nx), (nx, 1)
        else:
            shape, strides = (ny, nx, nz), (nx, 1, ny * nx)
        t = torch.as_tensor(_Buf(p.value, shape, strides, self), device="cuda")
        self._views[name] = t
        return t

    @property
    def r_E(self):
        return self._view("r_E")

    @property
    def f_E(self):
        return self._view("f_E")

    @property
    def delta_E(self):
        return self._view("delta_E")

    @property
    def H_prev(self):
        return self._view("H_prev")

    # -- configuration ---------------------------------------------------
    def _push_config(self):
        c = self.smoother_config
        f = self.enthalpy_forcing
        cfg = _lib.EnthalpyConfig(omega=float(c.omega), n_newton=int(c.n_newton), relaxation=float(c.relaxation),
                                  relative_tolerance=float(c.relative_tolerance),
                                  absolute_tolerance=float(c.absolute_tolerance), lf_c=float(c.lf_c),
                                  drain_rate=float(f.drain_rate.value), h_thin=float(f.h_thin.value),
                                  term_flags=int(self.term_flags.bitmask))
        _ecall("glide_enthalpy_set_config", self._h, ctypes.byref(cfg))

    def _bind(self, vel_div=None):
        """Point the kernels at the grid's thickness and the velocity source."""
        if vel_div is not None:
            self._vel_div = float(vel_div)
        H = self.grid.state.H.data
        inp = _lib.EnthalpyInputs()
        inp.H = ctypes.c_void_p(H.data_ptr())
        inp.ld_H = H.stride(0)
        if self._broadcast:
            u, v = self.grid.state.u.data, self.grid.state.v.data
            inp.u, inp.ld_u, inp.u_layer = ctypes.c_void_p(u.data_ptr()), u.stride(0), 0
            inp.v, inp.ld_v, inp.v_layer = ctypes.c_void_p(v.data_ptr()), v.stride(0), 0
        inp.vel_div = self._vel_div
        _ecall("glide_enthalpy_set_inputs", self._h, ctypes.byref(inp))

    def set_tuning(self, point_blocks_per_sm=None, column_blocks_per_sm=None, column_prefers_l1=None,
                   column_kernel=None):
        """Launch shapes of the kernels (no counterpart in the reference).
        column_kernel: "smem" (default; on-chip factors, 6 blocks of 64
        threads per SM), "smem8" (the same at 8 blocks per SM) or "local"
        (per-thread arrays)."""
        if column_kernel is not None:
            _ecall("glide_enthalpy_set_tuning", self._h, _lib.ENTH_TUNE_COLUMN_KERNEL,
                   {"local": 0, "smem": 1, "smem8": 2}[column_kernel])
        if point_blocks_per_sm is not None:
            _ecall("glide_enthalpy_set_tuning", self._h, _lib.ENTH_TUNE_POINT_BLOCKS, int(point_blocks_per_sm))
        if column_blocks_per_sm is not None:
            _ecall("glide_enthalpy_set_tuning", self._h, _lib.ENTH_TUNE_COLUMN_BLOCKS, int(column_blocks_per_sm))
        if column_prefers_l1 is not None:
            _ecall("glide_enthalpy_set_tuning", self._h, _lib.ENTH_TUNE_COLUMN_L1, int(bool(column_prefers_l1)))

    def counters(self):
        """(kernels launched, their algorithmic bytes) so far on this
        handle (glide_enthalpy_counters; instrumentation)."""
        n, b = ctypes.c_longlong(), ctypes.c_double()
        _ecall("glide_enthalpy_counters", self._h, ctypes.byref(n), ctypes.byref(b))
        return n.value, b.value

    def _materialize_velocity(self):
        if not self._broadcast:
            return
        u, v = self.grid.state.u.data, self.grid.state.v.data
        div = self._vel_div
        self._broadcast = False
        self._vel_div = 1.0
        self._bind()
        self._view("u3d")[:] = (u / div if div != 1.0 else u).unsqueeze(0)
        self._view("v3d")[:] = (v / div if div != 1.0 else v).unsqueeze(0)

    # -- operators --------------------------------------------------------
    def broadcast_velocity(self):
        """Use the grid's depth-averaged u, v for every sigma layer
        (glide/enthalpy.py:289-301), read in place: no layer copies."""
        self._broadcast = True
        self._vel_div = 1.0
        self._bind()

    def compute_omega(self, dh_dt, bmb=None):
        """omega = H sigma_dot from the sigma-space continuity equation
        (glide/enthalpy.py:303-339); dh_dt in the velocity's units."""
        self._push_config()
        self._bind()
        dh = torch.as_tensor(dh_dt, dtype=torch.float64, device="cuda").contiguous()
        b = None if bmb is None else torch.as_tensor(bmb, dtype=torch.float64, device="cuda").contiguous()
        _ecall("glide_enthalpy_compute_omega", self._h, ctypes.c_void_p(dh.data_ptr()), dh.stride(0),
               ctypes.c_void_p(b.data_ptr()) if b is not None else None, b.stride(0) if b is not None else 0,
               1.0, 1.0, _stream())

    def _prep(self):
        self._push_config()
        self._bind()

    def compute_residual(self, dt):
        """Residual at every node into r_E; returns max |r_E| (glide/enthalpy.py:341-364)."""
        self._prep()
        out = ctypes.c_double()
        _ecall("glide_enthalpy_residual", self._h, float(dt), 1, ctypes.byref(out), _stream())
        return out.value

    def column_smooth(self, dt):
        """One column Newton/Thomas smoother application into delta_E (glide/enthalpy.py:366-393)."""
        self._prep()
        _ecall("glide_enthalpy_column_smooth", self._h, float(dt), _stream())

    def layer_smooth(self, dt):
        """One pointwise Jacobi application into delta_E (glide/enthalpy.py:395-424)."""
        self._prep()
        _ecall("glide_enthalpy_layer_smooth", self._h, float(dt), _stream())

    def column_sweep(self, dt, n_iter, alternating=True):
        """Repeated smoothing with the reference's stop test (glide/enthalpy.py:426-471).
        Without a hook the whole loop runs on the device (one synchronisation)."""
        cfg = self.smoother_config
        if cfg.hook_func is not _no_hook:
            r0 = float(self.compute_residual(dt))
            if cfg.report_norms:
                print(f"  Enthalpy initial: |r0| = {r0:.2e}")
            for iteration in range(n_iter):
                self.column_smooth(dt)
                self.enthalpy_state.E[:] += cfg.omega * self.delta_E
                if alternating:
                    self.layer_smooth(dt)
                    self.enthalpy_state.E[:] += cfg.omega * self.delta_E
                cfg.hook_func(iteration)
                r = float(self.compute_residual(dt))
                rel = r / r0 if r0 > 0 else 0.0
                if cfg.report_norms:
                    print(f"  Enthalpy sweep {iteration}: |r|/|r0| = {rel:.2e}, |r| = {r:.2e}")
                if rel < cfg.relative_tolerance or r < cfg.absolute_tolerance:
                    break
            return
        self._prep()
        st = _lib.EnthalpyStats()
        _ecall("glide_enthalpy_column_sweep", self._h, float(dt), int(n_iter), int(bool(alternating)),
               ctypes.byref(st), _stream())
        self.last_stats = st
        if cfg.report_norms:
            print(f"  Enthalpy initial: |r0| = {st.initial_norm:.2e}")
            for it in range(min(st.iterations, len(st.history))):
                r = st.history[it]
                rel = r / st.initial_norm if st.initial_norm > 0 else 0.0
                print(f"  Enthalpy sweep {it}: |r|/|r0| = {rel:.2e}, |r| = {r:.2e}")

    def snapshot(self):
        """E_prev <- E, H_prev <- H."""
        self._bind()
        _ecall("glide_enthalpy_snapshot", self._h, _stream())

    def set_rhs(self, snapshot=True):
        """Precompute f_E (glide/enthalpy.py:473-519)."""
        if snapshot:
            self.snapshot()
        self._bind()
        _ecall("glide_enthalpy_set_rhs", self._h, _stream())

    # -- conversions (host-side formulas of glide/enthalpy.py:521-643) -----
    def set_surface_enthalpy_from_temperature(self, T_surface):
        T = torch.as_tensor(T_surface, dtype=torch.float64, device="cuda")
        T = torch.minimum(T, torch.tensor(T_MELT, dtype=torch.float64, device="cuda"))
        self._view("E_surface")[:] = C_I * (T - T_REF) / E_SCALE

    def _depth(self, k):
        return (1.0 - float(self.sigma[k])) * self.grid.state.H.data

    def initialize_from_temperature(self, T_field):
        ny, nx, nz = self.grid.ny, self.grid.nx, self.nz
        T = torch.as_tensor(T_field, dtype=torch.float64, device="cuda")
        if T.ndim == 0:
            T = torch.full((ny, nx, nz), float(T.item()), dtype=torch.float64, device="cuda")
        elif T.ndim == 2:
            T = T[:, :, None].expand(ny, nx, nz).clone()
        else:
            T = T.clone()
        for k in range(nz):
            T_pmp = T_MELT - BETA_CC * RHO_I * GRAVITY * self._depth(k)
            T[:, :, k] = torch.minimum(T[:, :, k], T_pmp)
        self.enthalpy_state.E[:] = C_I * (T - T_REF) / E_SCALE
        self.enthalpy_state.E_prev[:] = self.enthalpy_state.E
        self.H_prev[:] = self.grid.state.H.data

    def get_temperature(self):
        E = self.enthalpy_state.E
        T = torch.zeros(E.shape, dtype=torch.float64, device="cuda")
        for k in range(self.nz):
            T_pmp = T_MELT - BETA_CC * RHO_I * GRAVITY * self._depth(k)
            T[:, :, k] = torch.minimum(E[:, :, k] * E_SCALE / C_I + T_REF, T_pmp)
        return T

    def get_water_content(self):
        E = self.enthalpy_state.E
        w = torch.zeros(E.shape, dtype=torch.float64, device="cuda")
        for k in range(self.nz):
            w[:, :, k] = water_content_from_enthalpy(E[:, :, k] * E_SCALE, self._depth(k))
        return w

    def get_arrhenius_factor(self, out=None, scale=1.0):
        """Depth-averaged B = mean_k A(T, water)^(-1/n) (glide/enthalpy.py:600-643),
        divided by `scale`; written into `out` (any (ny, nx) float64 view) when given."""
        self._bind()
        if out is None:
            out = torch.empty((self.grid.ny, self.grid.nx), dtype=torch.float64, device="cuda")
        if out.stride(1) != 1:
            raise ValueError("out must have unit column stride")
        n = float(self.grid.rheology.n.value)
        _ecall("glide_enthalpy_arrhenius", self._h, n, float(scale), ctypes.c_void_p(out.data_ptr()),
               out.stride(0), _stream())
        return out


class _StateView:
    def __init__(self, ops):
        self._ops = ops

    @property
    def E(self):
        return self._ops._view("E")

    @property
    def E_prev(self):
        return self._ops._view("E_prev")

    def __repr__(self):
        return f"EnthalpyState: E {tuple(self.E.shape)}"


class _ForcingView:
    def __init__(self, ops):
        self._ops = ops
        base = EnthalpyForcing()
        self.drain_rate = base.drain_rate
        self.h_thin = base.h_thin

    @property
    def E_surface(self):
        return self._ops._view("E_surface")

    @property
    def Q_geo(self):
        return self._ops._view("Q_geo")

    @property
    def Q_fh(self):
        return self._ops._view("Q_fh")

    @property
    def phi_strain(self):
        return self._ops._view("phi_strain")
