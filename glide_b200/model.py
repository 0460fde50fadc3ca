"""Model API (mirror of glide/model.py:24-94): `IceDynamics` forward/backward."""
from __future__ import annotations

import torch

from . import _lib
from .multigrid import FASAdjointSolver, FASCDSolver, Multigrid


class IceDynamics:
    """Momentum + mass conservation (SSA) on a multigrid hierarchy."""

    def __init__(self, mg: Multigrid | None = None, n_levels=None, grid=None, ny=None, nx=None, dx=None,
                 x0=0.0, y0=0.0, crs=None, dtype=torch.float64, reference_quirks=True):
        if mg is not None:
            self.mg = mg
        elif grid is not None and n_levels is not None:
            self.mg = Multigrid(n_levels, finest_grid=grid, reference_quirks=reference_quirks)
        elif ny and nx and dx and n_levels:
            self.mg = Multigrid(n_levels, ny=ny, nx=nx, dx=dx, x0=x0, y0=y0, crs=crs, dtype=dtype,
                                reference_quirks=reference_quirks)
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
        (glide/model.py:74-94)."""
        h = self.mg.hierarchy
        top = self.top_level
        for name, g in (("adj_f_u", dJdu), ("adj_f_v", dJdv), ("adj_f_H", dJdH)):
            if g is None:
                h.set(name, top, 0.0)
            else:
                h.set(name, top, -torch.as_tensor(g, device="cuda", dtype=h.dtype))
        mask = ((_lib.GRAD_BETA if compute_beta_grad else 0) | (_lib.GRAD_BED if compute_bed_grad else 0) |
                (_lib.GRAD_H_PREV if compute_H_prev_grad else 0) | (_lib.GRAD_SMB if compute_smb_grad else 0))
        return self.adjoint_solver.solve(dt, start_level=top, grad_mask=mask)
