"""One level of the MAC-grid hierarchy (mirror of glide/grid.py).

A `Grid` is a view of level `level` of a device `Hierarchy`: its Fields alias
the arena and its Constants push to the level's physical parameters.  A
stand-alone `Grid(ny, nx, dx)` owns a one-level hierarchy.
Defaults and units restate glide/grid.py:8-145; layout glide/grid.py:167-217.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from .field import Constant, Field, GridEntity, SubgridField
from .hierarchy import Hierarchy
from .operators import AdjointOperators, ForwardOperators


@dataclass
class State:
    u: Field = None
    v: Field = None
    H: Field = None
    H_prev: Field = None
    phi: Field = None
    mask: Field = None

    def __repr__(self):
        return "\n".join(f.compact_string for f in (self.u, self.v, self.H, self.H_prev, self.phi, self.mask))


@dataclass
class AdjointState:
    lambda_u: Field = None
    lambda_v: Field = None
    lambda_H: Field = None


@dataclass
class Geometry:
    bed: SubgridField = None
    thklim: Constant = None
    flotation_reg_driving: Constant = None


@dataclass
class Rheology:
    B: Field = None
    n: Constant = None
    eps_reg: Constant = None


@dataclass
class Sliding:
    beta: Field = None
    m: Constant = None
    u_reg: Constant = None
    water_drag: Constant = None
    flotation_reg_sliding: Constant = None


@dataclass
class Calving:
    calving_rate: Constant = None
    flotation_reg_calving: Constant = None


@dataclass
class Forcing:
    smb: Field = None


class Grid:
    """Single level of the multigrid hierarchy (glide/grid.py:147-372)."""

    def __init__(self, ny: int = None, nx: int = None, dx: float = None, x0: float = 0.0, y0: float = 0.0,
                 crs=None, parent=None, *, hierarchy: Hierarchy | None = None, level: int = 0,
                 dtype=torch.float64):
        if hierarchy is None:
            hierarchy = Hierarchy(ny, nx, dx, 1, dtype=dtype)
            level = 0
        self._hier = hierarchy
        self.level = level
        self.ny, self.nx, self.dx = hierarchy.shapes[level]
        self.parent = parent
        self.child = None
        self.x0, self.y0 = float(x0), float(y0)
        self.crs = crs
        dx = self.dx
        dev = "cuda"
        self.x_cell = self.x0 + dx * torch.arange(self.nx, device=dev, dtype=torch.float64)
        self.y_cell = self.y0 - dx * torch.arange(self.ny, device=dev, dtype=torch.float64)
        self.x_vfacet = self.x0 - dx / 2 + dx * torch.arange(self.nx + 1, device=dev, dtype=torch.float64)
        self.y_hfacet = self.y0 + dx / 2 - dx * torch.arange(self.ny + 1, device=dev, dtype=torch.float64)
        self.nu = self.ny * (self.nx + 1)
        self.nv = (self.ny + 1) * self.nx
        self.nh = self.ny * self.nx
        self.n_total = self.nu + self.nv + self.nh

        def F(name, ent, units, grad=None, cls=Field):
            return cls(hierarchy, name, level, ent, dx, grid=self, units=units, grad_name=grad)

        C, VF, HF = GridEntity.CELL, GridEntity.VERTICAL_FACET, GridEntity.HORIZONTAL_FACET
        phys = hierarchy.get_phys(level)

        def K(name, units):
            return Constant(phys[name], name=name, units=units,
                            on_set=lambda v, n=name: hierarchy.set_phys(level, **{n: v}))

        self.state = State(u=F("u", VF, "m a^{-1}"), v=F("v", HF, "m a^{-1}"), H=F("H", C, "m"),
                           H_prev=F("H_prev", C, "m", grad="grad_H_prev"), phi=F("phi", C, ""),
                           mask=F("mask", C, ""))
        self.geometry = Geometry(bed=F("bed", C, "m", grad="grad_bed", cls=SubgridField),
                                 thklim=K("thklim", "m"),
                                 flotation_reg_driving=K("flotation_reg_driving", "m^{-1}"))
        self.rheology = Rheology(B=F("B", C, ""), n=K("n", ""), eps_reg=K("eps_reg", "s^{-2}"))
        self.sliding = Sliding(beta=F("beta", C, "", grad="grad_beta"), m=K("m", ""),
                               u_reg=K("u_reg", "m a^{-1}"), water_drag=K("water_drag", ""),
                               flotation_reg_sliding=K("flotation_reg_sliding", "m"))
        self.calving = Calving(calving_rate=K("calving_rate", "m a^{-1}"),
                               flotation_reg_calving=K("flotation_reg_calving", "m"))
        self.forcing = Forcing(smb=F("smb", C, "m a^{-1}", grad="grad_smb"))
        self._adjoint = None
        self._forward_operators = None
        self._adjoint_operators = None

    @property
    def adjoint(self) -> AdjointState:
        if self._adjoint is None:
            h, l, dx = self._hier, self.level, self.dx
            self._adjoint = AdjointState(
                lambda_u=Field(h, "lambda_u", l, GridEntity.VERTICAL_FACET, dx, grid=self),
                lambda_v=Field(h, "lambda_v", l, GridEntity.HORIZONTAL_FACET, dx, grid=self),
                lambda_H=Field(h, "lambda_H", l, GridEntity.CELL, dx, grid=self))
        return self._adjoint

    @property
    def forward_operators(self) -> ForwardOperators:
        if self._forward_operators is None:
            self._forward_operators = ForwardOperators(self)
        return self._forward_operators

    @property
    def adjoint_operators(self) -> AdjointOperators:
        if self._adjoint_operators is None:
            self._adjoint_operators = AdjointOperators(self)
        return self._adjoint_operators

    def spawn_child(self):
        """A new stand-alone Grid of half the cells and twice the spacing,
        linked as this grid's child, fields zero (glide/grid.py:374-380; the
        reference leaves the origin at 0, as here)."""
        child = Grid(self.ny // 2, self.nx // 2, self.dx * 2, parent=self, dtype=self._hier.dtype)
        self.child = child
        return child

    def __repr__(self):
        return f"Grid(level={self.level}, ny={self.ny}, nx={self.nx}, dx={self.dx})"
