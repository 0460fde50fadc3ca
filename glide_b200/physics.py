"""`IcePhysics`: the README-level facade of the reference (README.md:31-50),
over `IceDynamics`.

    phys = IcePhysics(ny, nx, dx, n_levels)
    phys.set_geometry(bed, thickness)
    phys.set_parameters(B, beta, smb)
    u, v, H = phys.forward(dt, n_vcycles)
    grad_beta = phys.adjoint(dL_du, dL_dv)
"""
from __future__ import annotations

import torch

from .model import IceDynamics


class IcePhysics:
    def __init__(self, ny: int, nx: int, dx: float, n_levels: int, dtype=torch.float64,
                 reference_quirks: bool = True):
        self.model = IceDynamics(n_levels=n_levels, ny=ny, nx=nx, dx=dx, dtype=dtype,
                                 reference_quirks=reference_quirks)
        self.mg = self.model.mg
        self._dt = None

    def set_geometry(self, bed, thickness):
        self.mg.geometry.bed.set(bed)
        self.mg.state.H.set(thickness)
        self.mg.state.H_prev.set(thickness)

    def set_parameters(self, B, beta, smb):
        self.mg.rheology.B.set(B)
        self.mg.sliding.beta.set(beta)
        self.mg.forcing.smb.set(smb)

    def forward(self, dt: float, n_vcycles: int = 10, relative_tolerance: float = 0.0,
                absolute_tolerance: float = 0.0, update_geometry: bool = False):
        """Run up to `n_vcycles` FASCD V-cycles for one step of length dt.
        Returns new tensors (u, v, H) of the finest level."""
        s = self.model.forward_solver
        s.fas_options.set(maximum_vcycles=int(n_vcycles), relative_tolerance=relative_tolerance,
                          absolute_tolerance=absolute_tolerance, report_norms=False)
        self._dt = float(dt)
        self.model.forward(0.0, dt, update_geometry=update_geometry)
        st = self.mg[0].state
        return st.u.data.clone(), st.v.data.clone(), st.H.data.clone()

    def adjoint(self, dL_du, dL_dv, dL_dH=None, n_vcycles: int = 10):
        """Gradient of a loss L(u, v, H) with respect to beta at the last forward
        state.  Returns a new tensor (ny, nx)."""
        if self._dt is None:
            raise RuntimeError("call forward() before adjoint()")
        a = self.model.adjoint_solver
        a.fas_options.set(maximum_vcycles=int(n_vcycles), relative_tolerance=0.0, absolute_tolerance=0.0,
                          report_norms=False)
        self.model.backward(0.0, self._dt, dJdu=dL_du, dJdv=dL_dv, dJdH=dL_dH)
        return self.mg[0].sliding.beta.grad.clone()
