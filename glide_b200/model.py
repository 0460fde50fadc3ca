"""Model API (mirror of glide/model.py:24-94): `IceDynamics` forward/backward."""
from __future__ import annotations

import torch

from . import _lib
from .multigrid import FASAdjointSolver, FASCDSolver, Multigrid


class IceDynamics:
    """Momentum + mass conservation (SSA) on a multigrid hierarchy."""

    def __init__(self, mg: Multigrid | None = None, n_levels=None, grid=None, ny=None, nx=None, dx=None,
                 x0=0.0, y0=0.0, crs=None, dtype=torch.float64, reference_quirks=True, precision=None):
        """precision: None (from dtype), "fp64", "fp32" or "mixed" (binary64
        state and residual, binary32 smoother and tangent multigrid)."""
        if mg is not None:
            self.mg = mg
        elif grid is not None and n_levels is not None:
            self.mg = Multigrid(n_levels, finest_grid=grid, reference_quirks=reference_quirks, precision=precision)
        elif ny and nx and dx and n_levels:
            self.mg = Multigrid(n_levels, ny=ny, nx=nx, dx=dx, x0=x0, y0=y0, crs=crs, dtype=dtype,
                                reference_quirks=reference_quirks, precision=precision)
        else:
            raise ValueError("Must supply either (a) a multigrid object (b) a grid and number of levels "
                             "(c) ny/nx/dx and number of levels")
        self._forward_solver = None
        self._adjoint_solver = None
        self.top_level = 0
        self._post_forward_hooks = []

    @property
    def forward_solver(self) -> FASCDSolver:
        if self._forward_solver is None:
            self._forward_solver = FASCDSolver(self.mg)
        return self._forward_solver

    @property
    def adjoint_solver(self) -> FASAdjointSolver:
        if self._adjoint_solver is None:
            self._adjoint_solver = FASAdjointSolver(self.mg)
        return self._adjoint_solver

    def set_top_level(self, level):
        self.top_level = level

    def register_post_forward_hook(self, hook):
        self._post_forward_hooks.append(hook)

    def forward(self, t, dt, update_geometry=True):
        """One implicit time step: solve for u, v, H at t + dt (glide/model.py:65-72)."""
        st = self.forward_solver.solve(dt, start_level=self.top_level)
        if update_geometry:
            lev = self.mg.levels[self.top_level]
            lev.state.H_prev.data.copy_(lev.state.H.data)
        for f in self._post_forward_hooks:
            f(t + dt)
        return st

    def backward(self, t, dt, dJdu=None, dJdv=None, dJdH=None, compute_beta_grad=True,
                 compute_bed_grad=True, compute_H_prev_grad=True, compute_smb_grad=True):
        """Adjoint solve with forcing -dJ/dx, then the parameter gradients
        (glide/model.py:74-94).

        The reference starts each adjoint solve from the previous lambda.  Its
        lambda on the Dirichlet faces is left unconstrained by the adjoint
        residual yet enters the gradient kernels, so a gradient depends on
        which solve ran before it.  Reference mode keeps that; native mode
        (reference_quirks=False) starts every solve from lambda = 0, which
        makes each gradient a function of this step's inputs alone."""
        mask = self.prepare_backward(dJdu, dJdv, dJdH, compute_beta_grad, compute_bed_grad, compute_H_prev_grad,
                                     compute_smb_grad)
        return self.adjoint_solver.solve(dt, start_level=self.top_level, grad_mask=mask)

    def prepare_backward(self, dJdu=None, dJdv=None, dJdH=None, compute_beta_grad=True, compute_bed_grad=True,
                         compute_H_prev_grad=True, compute_smb_grad=True) -> int:
        """The adjoint solve's inputs as `backward` sets them (right-hand side
        -dJ/dx, lambda = 0 in native mode); returns the gradient mask.  For
        grouped solves (glide_b200.group), which then solve many members at
        once."""
        h = self.mg.hierarchy
        top = self.top_level
        if not getattr(h, "reference_quirks", True):
            for name in ("lambda_u", "lambda_v", "lambda_H"):
                h.set(name, top, 0.0, restrict_down=True)
        for name, g in (("adj_f_u", dJdu), ("adj_f_v", dJdv), ("adj_f_H", dJdH)):
            if g is None:
                h.set(name, top, 0.0)
            else:
                h.set(name, top, -torch.as_tensor(g, device="cuda", dtype=h.dtype))
        return ((_lib.GRAD_BETA if compute_beta_grad else 0) | (_lib.GRAD_BED if compute_bed_grad else 0) |
                (_lib.GRAD_H_PREV if compute_H_prev_grad else 0) | (_lib.GRAD_SMB if compute_smb_grad else 0))


class ThermalModel:
    """Enthalpy solver coupled to the momentum solve (mirror of glide/model.py:97-281).

    step(dt): omega from the realised thickness change, frictional heating,
    forcing, column sweeps, then the depth-averaged rate factor fed back into
    the grid's B.  In reference mode (the hierarchy's reference quirks on)
    only that grid's B changes and coarser levels keep theirs, as in the
    reference (glide/model.py:216-222).  In native mode the new B is also
    restricted to every coarser level, so the coarse-grid corrections of the
    next momentum solve use the same viscosity as the fine level; with stale
    coarse B a large change of the rate factor stalls the multigrid solve.
    The SSA velocity is read in place for every sigma layer (no layer copies);
    the m/a -> m/s conversion is applied by the kernels as they read it.
    """

    SEC_PER_YR = 365.25 * 86400.0

    def __init__(self, grid, nz=21, n_smooth=10, update_rheology=True, frictional_heating=True, rho_i=917.0):
        from .enthalpy import EnthalpyOperators
        self.ops = EnthalpyOperators(grid, nz=nz)
        self.n_smooth = n_smooth
        self.update_rheology = update_rheology
        self.frictional_heating = frictional_heating
        self.rho_i = rho_i
        self.g = 9.81

    def initialize(self, T_surface, T_field=None, Q_geo=None):
        """Initial temperature, surface Dirichlet data and geothermal flux (glide/model.py:134-153)."""
        if T_field is None:
            T_field = T_surface
        self.ops.initialize_from_temperature(T_field)
        self.ops.set_surface_enthalpy_from_temperature(T_surface)
        if Q_geo is not None:
            self.ops.enthalpy_forcing.Q_geo[:] = torch.as_tensor(Q_geo, dtype=torch.float64, device="cuda")

    def pre_momentum(self):
        """Snapshot E and H before the momentum step (glide/model.py:155-164)."""
        self.ops.snapshot()

    def step(self, dt):
        """Advance enthalpy by dt seconds (glide/model.py:166-222)."""
        from .enthalpy import _ecall, _stream
        import ctypes
        ops = self.ops
        sec = self.SEC_PER_YR
        ops._push_config()
        ops.broadcast_velocity()
        # omega in m/a from (H - H_prev) / dt_yr, then converted to m/s
        dt_yr = dt / sec
        _ecall("glide_enthalpy_compute_omega", ops._h, None, 0, None, 0, float(dt_yr), float(sec), _stream())
        ops._bind(vel_div=sec)
        if self.frictional_heating:
            sl = ops.grid.sliding
            beta = sl.beta.data
            _ecall("glide_enthalpy_frictional_heating", ops._h, ctypes.c_void_p(beta.data_ptr()), beta.stride(0),
                   float(sl.m.value), float(sl.u_reg.value), _stream())
        ops.set_rhs(snapshot=False)
        ops.column_sweep(dt, self.n_smooth)
        if self.update_rheology:
            n = float(ops.grid.rheology.n.value)
            scale = self.rho_i * self.g * sec ** (1.0 / n)
            ops.get_arrhenius_factor(out=ops.grid.rheology.B.data, scale=scale)
            hier = getattr(ops.grid, "_hier", None)
            if hier is not None and not getattr(hier, "reference_quirks", True):
                hier.restrict("B", ops.grid.level)

    @property
    def B_scale(self):
        n = float(self.ops.grid.rheology.n.value)
        return self.rho_i * self.g * self.SEC_PER_YR ** (1.0 / n)

    @property
    def temperature(self):
        return self.ops.get_temperature()

    @property
    def water_content(self):
        return self.ops.get_water_content()

    @property
    def enthalpy(self):
        return self.ops.enthalpy_state.E

    @property
    def sigma(self):
        return self.ops.sigma
