"""Multi-level inversion for the basal traction beta.

The driver of the reference's inverse examples
(examples/greenland/greenland_inverse.py:71-175), as a library routine:

* the velocity observations are restricted down the hierarchy with 2 x 2
  cell averages (`observation_hierarchy`, the example's :71-76);
* log beta is optimised level by level, coarsest first: every epoch runs one
  `GlideStep` (forward solve) at that level, evaluates the masked L1
  velocity misfit plus Tikhonov and total-variation penalties on log beta,
  and back-propagates through the adjoint solve (the example's :103-166);
* between levels log beta is prolongated bilinearly (:172-173).

Solver options are the caller's: set `model.forward_solver.fas_options` and
`model.adjoint_solver.fas_options` before calling, as the example does.
I/O (the example's VTI/NetCDF writers) is left to the `callback`.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import torch

from .torch import GlideStep


def observation_hierarchy(mg, u_obs, v_obs, n_levels: int | None = None):
    """[(u_obs, v_obs) at level 0, level 1, ...]: cell-centred velocities
    restricted with 2 x 2 averages (glide/multigrid.py restrict_cell)."""
    n_levels = mg.n_levels if n_levels is None else n_levels
    u = torch.as_tensor(u_obs, device="cuda", dtype=mg.hierarchy.dtype)
    v = torch.as_tensor(v_obs, device="cuda", dtype=mg.hierarchy.dtype)
    levels = [(u, v)]
    for _ in range(1, n_levels):
        u, v = mg.restrict_cell(levels[-1][0]), mg.restrict_cell(levels[-1][1])
        levels.append((u, v))
    return levels


@dataclass
class InversionLoss:
    """J = J_data + J_L1 + J_L2 of the reference example
    (greenland_inverse.py:131-155): masked L1 misfit of the cell-centred
    velocity, plus l2 * sum |grad log beta|^2 dx^2 and
    tv * sum sqrt(|grad log beta|^2 + eps^2) dx^2."""
    l2: float = 1e-5
    tv: float = 1e-8
    eps: float = 1e-6
    mask_threshold: float = 0.01

    def __call__(self, u, v, u_obs, v_obs, log_beta, dx):
        u_cell = 0.5 * (u[:, 1:] + u[:, :-1])
        v_cell = 0.5 * (v[1:] + v[:-1])
        u_mask = u_obs.abs() > self.mask_threshold
        v_mask = v_obs.abs() > self.mask_threshold
        j_data = ((u_cell - u_obs).abs() * u_mask).mean() + ((v_cell - v_obs).abs() * v_mask).mean()
        gy = torch.diff(log_beta, dim=0) / dx
        gx = torch.diff(log_beta, dim=1) / dx
        j_l2 = self.l2 * ((gy ** 2).sum() + (gx ** 2).sum()) * dx ** 2
        j_l1 = self.tv * torch.sqrt(gy[:, :-1] ** 2 + gx[:-1] ** 2 + self.eps ** 2).sum() * dx ** 2
        return j_data + j_l1 + j_l2, j_data, j_l1, j_l2


@dataclass
class InversionResult:
    log_beta: torch.Tensor                       # at level 0 (or the finest level solved)
    history: list = field(default_factory=list)  # (level, epoch, J, J_data, J_L1, J_L2)


def invert_beta(model, u_obs, v_obs, dt: float, coarsest_level: int | None = None, epochs_per_level: int = 50,
                loss: InversionLoss | None = None,
                optimizer: Callable[[list], torch.optim.Optimizer] | None = None,
                log_beta: torch.Tensor | None = None, t: float = 0.0,
                callback: Callable[[int, int, dict], None] | None = None) -> InversionResult:
    """Optimise log beta from `coarsest_level` down to level 0.

    u_obs, v_obs: cell-centred observed velocities at level 0.  The start is
    log of the model's beta at `coarsest_level` unless `log_beta` is given
    there.  `optimizer(params)` builds the optimiser of each level (default
    RMSprop with lr 1e-2, the example's choice).  `callback(level, epoch,
    terms)` runs after every epoch."""
    mg = model.mg
    coarsest_level = mg.n_levels - 1 if coarsest_level is None else coarsest_level
    loss = loss or InversionLoss()
    optimizer = optimizer or (lambda params: torch.optim.RMSprop(params, lr=1e-2))
    obs = observation_hierarchy(mg, u_obs, v_obs, coarsest_level + 1)
    if log_beta is None:
        log_beta = torch.log(mg[coarsest_level].sliding.beta.data.clone())
    log_beta = log_beta.detach().clone()
    result = InversionResult(log_beta=log_beta)
    for level in range(coarsest_level, -1, -1):
        log_beta.requires_grad_(True)
        grid = mg[level]
        H_prev = grid.state.H_prev.data.detach().clone()
        bed = grid.geometry.bed.data.detach().clone()
        smb = grid.forcing.smb.data.detach().clone()
        u_o, v_o = obs[level]
        opt = optimizer([log_beta])
        for epoch in range(epochs_per_level):
            opt.zero_grad()
            beta = torch.exp(log_beta)
            u, v, _H = GlideStep.apply(t, dt, model, level, H_prev, bed, beta, smb)
            J, j_data, j_l1, j_l2 = loss(u, v, u_o, v_o, log_beta, grid.dx)
            J.backward()
            opt.step()
            terms = {"J": J.item(), "J_data": j_data.item(), "J_L1": j_l1.item(), "J_L2": j_l2.item()}
            result.history.append((level, epoch, terms["J"], terms["J_data"], terms["J_L1"], terms["J_L2"]))
            if callback is not None:
                callback(level, epoch, terms)
        log_beta = log_beta.detach()
        if level > 0:
            log_beta = mg.prolongate_cell(log_beta.contiguous(), method="bilinear")
    model.set_top_level(0)
    result.log_beta = log_beta
    return result
