"""Multigrid hierarchy, field managers and the FASCD / FASAdjoint solvers
(mirror of glide/multigrid.py).

The V-cycle schedules themselves (glide/multigrid.py:502-645 and :873-973)
run inside libglide_b200.so; these classes keep the reference's Python
surface: the field managers that set a field on a level and restrict it down
(glide/multigrid.py:264-484), the option objects with key validation
(:687-1071) and `solve`.
"""
from __future__ import annotations

from dataclasses import dataclass, fields

import torch

from .field import BroadcastOption, LocalOption
from .grid import Grid
from .hierarchy import Hierarchy
from .operators import NewtonConfig, VankaConfig, _Synced


class Multigrid:
    """Level hierarchy (glide/multigrid.py:8-116).  ny, nx must be divisible by
    2^(n_levels-1); every level halves the previous one and doubles dx."""

    def __init__(self, n_levels: int, finest_grid: Grid | None = None, ny=None, nx=None, dx=None,
                 x0=0.0, y0=0.0, crs=None, use_fast_math=True, dtype=torch.float64,
                 reference_quirks: bool = True, use_graphs: bool = True, precision: str | None = None):
        if finest_grid is not None:
            ny, nx, dx = finest_grid.ny, finest_grid.nx, finest_grid.dx
            x0, y0, crs = finest_grid.x0, finest_grid.y0, finest_grid.crs
            dtype = finest_grid._hier.dtype
        self.hierarchy = Hierarchy(ny, nx, dx, n_levels, dtype=dtype, reference_quirks=reference_quirks,
                                   use_graphs=use_graphs, precision=precision)
        self.n_levels = n_levels
        self.levels = []
        for l in range(n_levels):
            d = dx * 2 ** l
            off = sum(dx * 2 ** k / 2 for k in range(l))
            g = Grid(hierarchy=self.hierarchy, level=l, x0=x0 + off, y0=y0 - off, crs=crs,
                     parent=self.levels[-1] if self.levels else None)
            if self.levels:
                self.levels[-1].child = g
            self.levels.append(g)
        if finest_grid is not None:
            for name in ("u", "v", "H", "H_prev", "phi", "mask", "bed", "B", "beta", "smb"):
                self.hierarchy.set(name, 0, finest_grid._hier.view(name, 0), restrict_down=True)
        self.finest_grid = self.levels[0]
        self.state = _Managers(self, {"u": "u", "v": "v", "H": "H", "H_prev": "H_prev", "phi": "phi",
                                      "mask": "mask"})
        self.geometry = _Managers(self, {"bed": "bed"}, {"thklim": "thklim",
                                                         "flotation_reg_driving": "flotation_reg_driving"})
        self.rheology = _Managers(self, {"B": "B"}, {"n": "n", "eps_reg": "eps_reg"})
        self.sliding = _Managers(self, {"beta": "beta"}, {"m": "m", "u_reg": "u_reg", "water_drag": "water_drag",
                                                         "flotation_reg_sliding": "flotation_reg_sliding"})
        self.calving = _Managers(self, {}, {"calving_rate": "calving_rate",
                                            "flotation_reg_calving": "flotation_reg_calving"})
        self.forcing = _Managers(self, {"smb": "smb"})
        self._adjoint = None

    @property
    def adjoint(self):
        if self._adjoint is None:
            self._adjoint = _Managers(self, {"lambda_u": "lambda_u", "lambda_v": "lambda_v",
                                             "lambda_H": "lambda_H"})
        return self._adjoint

    def __getitem__(self, key):
        return self.levels[key]


class HierarchyFieldManager:
    """Set a field on `start_level` and restrict it to every coarser level
    (glide/multigrid.py:264-283): face averages for u/v, 2x2 maximum for the
    mask, 2x2 average for other cell fields."""

    def __init__(self, mg: Multigrid, name: str):
        self._mg = mg
        self._name = name

    def set(self, value, start_level=0):
        self._mg.hierarchy.set(self._name, start_level, value, restrict_down=True)

    def restrict_down(self, start_level):
        self._mg.hierarchy.restrict(self._name, start_level)

    def set_level(self, level, value):
        self._mg.hierarchy.set(self._name, level, value, restrict_down=False)


class ConstantManager:
    """Set a scalar parameter on `start_level` and every coarser level."""

    def __init__(self, mg: Multigrid, name: str):
        self._mg = mg
        self._name = name

    def set(self, value, start_level=0):
        for l in range(start_level, self._mg.n_levels):
            getattr(_owner_of(self._mg.levels[l], self._name), self._name).set(value)

    def set_level(self, level, value):
        getattr(_owner_of(self._mg.levels[level], self._name), self._name).set(value)


def _owner_of(grid: Grid, name: str):
    for group in (grid.geometry, grid.rheology, grid.sliding, grid.calving):
        if hasattr(group, name):
            return group
    raise AttributeError(name)


class _Managers:
    def __init__(self, mg, fields_map, consts=None):
        self.mg = mg
        for attr, name in fields_map.items():
            setattr(self, attr, HierarchyFieldManager(mg, name))
        for attr, name in (consts or {}).items():
            setattr(self, attr, ConstantManager(mg, name))


# ----------------------------------------------------------------- options
@dataclass
class FASCDConfig(_Synced):
    """glide/multigrid.py:672-682."""
    freeze_coarse_calving: bool = True
    freeze_coarse_phi: bool = True
    coarsest_steps: int = 200
    pre_steps: int = 10
    post_steps: int = 20
    finest_steps: int = 50
    maximum_vcycles: int = 10
    relative_tolerance: float = 1e-3
    absolute_tolerance: float = 5.0
    report_norms: bool = True


@dataclass
class FASAdjointConfig(_Synced):
    """glide/multigrid.py:993-1001."""
    coarsest_steps: int = 200
    pre_steps: int = 10
    post_steps: int = 20
    finest_steps: int = 50
    maximum_vcycles: int = 10
    relative_tolerance: float = 1e-3
    absolute_tolerance: float = 5.0
    report_norms: bool = True


def validate_kwargs(config_cls, kwargs):
    """glide/multigrid.py:687-694."""
    valid = {f.name for f in fields(config_cls)}
    unknown = set(kwargs) - valid
    if unknown:
        raise AttributeError(f"Unknown {config_cls.__name__} option(s): {sorted(unknown)}. "
                             f"Valid options are: {sorted(valid)}")


def _bind_fas(cfg, hier, adjoint):
    def push():
        kw = dict(coarsest_steps=cfg.coarsest_steps, pre_steps=cfg.pre_steps, post_steps=cfg.post_steps,
                  finest_steps=cfg.finest_steps, maximum_vcycles=cfg.maximum_vcycles,
                  relative_tolerance=cfg.relative_tolerance, absolute_tolerance=cfg.absolute_tolerance)
        if not adjoint:
            kw.update(freeze_coarse_calving=int(cfg.freeze_coarse_calving),
                      freeze_coarse_phi=int(cfg.freeze_coarse_phi))
        hier.set_fas(adjoint, **kw)
    cfg._bind(push)
    push()


class _FasOptionsBase:
    _cls = None

    def __init__(self, config):
        self._config = config
        for f in fields(self._cls):
            setattr(self, f.name, LocalOption(getter=lambda n=f.name: getattr(self._config, n),
                                              setter=lambda v, n=f.name: setattr(self._config, n, v),
                                              name=f.name))

    def set(self, **kwargs):
        validate_kwargs(self._cls, kwargs)
        for k, v in kwargs.items():
            setattr(self._config, k, v)

    def __repr__(self):
        return "fas_options={" + ", ".join(repr(getattr(self, f.name)) for f in fields(self._cls)) + "}"


class FASCDOptions(_FasOptionsBase):
    """glide/multigrid.py:696-777."""
    _cls = FASCDConfig


class FASAdjointOptions(_FasOptionsBase):
    """glide/multigrid.py:1004-1071."""
    _cls = FASAdjointConfig


class VankaOptions:
    """Broadcast wrapper over every level's VankaConfig (glide/multigrid.py:780-815)."""

    def __init__(self, levels, getter):
        self._levels = levels
        self._getter = getter
        self.options = ["omega", "relax_phi"]
        self.omega = BroadcastOption(levels, getter, "omega")
        self.relax_phi = BroadcastOption(levels, getter, "relax_phi")
        self.newton_options = NewtonOptions(levels, lambda lev: getter(lev).newton_config)

    def set(self, **kwargs):
        validate_kwargs(VankaConfig, kwargs)
        for lev in self._levels:
            for k, v in kwargs.items():
                setattr(self._getter(lev), k, v)

    def set_level(self, level_index, **kwargs):
        validate_kwargs(VankaConfig, kwargs)
        for k, v in kwargs.items():
            setattr(self._getter(self._levels[level_index]), k, v)

    def __repr__(self):
        return "vanka_options={" + ", ".join(repr(getattr(self, o)) for o in self.options) + "}"


class NewtonOptions:
    """glide/multigrid.py:818-852."""

    def __init__(self, levels, getter):
        self._levels = levels
        self._getter = getter
        self.options = ["steps", "relaxation", "ssa_damping", "mc_damping"]
        for o in self.options:
            setattr(self, o, BroadcastOption(levels, getter, o))

    def set(self, **kwargs):
        validate_kwargs(NewtonConfig, kwargs)
        for lev in self._levels:
            for k, v in kwargs.items():
                setattr(self._getter(lev), k, v)

    def set_level(self, level_index, **kwargs):
        validate_kwargs(NewtonConfig, kwargs)
        for k, v in kwargs.items():
            setattr(self._getter(self._levels[level_index]), k, v)

    def __repr__(self):
        return "newton_options={" + ", ".join(repr(getattr(self, o)) for o in self.options) + "}"


@dataclass
class FASCDLevel:
    grid: Grid


class FASCDSolver:
    """Full Approximation Scheme with Constrained Descent for the coupled
    SSA + mass system (glide/multigrid.py:486-533)."""

    def __init__(self, multigrid: Multigrid):
        self.multigrid = multigrid
        self.levels = [FASCDLevel(g) for g in multigrid.levels]
        self._fas_config = FASCDConfig()
        _bind_fas(self._fas_config, multigrid.hierarchy, adjoint=False)
        self.fas_options = FASCDOptions(self._fas_config)
        self.vanka_options = VankaOptions(self.levels, lambda lev: lev.grid.forward_operators.vanka_config)
        self.n_levels = len(self.levels)
        self.dt = None
        self.last_stats = None

    def solve(self, dt, start_level=0, report_norms=True):
        self.dt = float(dt)
        st = self.multigrid.hierarchy.forward(float(dt), start_level)
        self.last_stats = st
        if self._fas_config.report_norms and report_norms:
            h = st["history"]
            print(f"  Initial:   |r0|     = {h[0]:.2e}")
            for k in range(1, len(h)):
                print(f"  V-cycle {k - 1}: |r|/|r0| = {h[k] / h[0]:.2e}")
        return st


@dataclass
class FASAdjointLevel:
    grid: Grid


class FASAdjointSolver:
    """Linear FAS on the adjoint system J^T lambda = -dJ/dx
    (glide/multigrid.py:857-903)."""

    def __init__(self, multigrid: Multigrid):
        self.multigrid = multigrid
        self.levels = [FASAdjointLevel(g) for g in multigrid.levels]
        self._fas_config = FASAdjointConfig()
        _bind_fas(self._fas_config, multigrid.hierarchy, adjoint=True)
        self.fas_options = FASAdjointOptions(self._fas_config)
        self.vanka_options = VankaOptions(self.levels, lambda lev: lev.grid.adjoint_operators.vanka_config)
        self.n_levels = len(self.levels)
        self.dt = None
        self.last_stats = None

    def solve(self, dt, start_level=0, report_norms=True, grad_mask=0):
        self.dt = float(dt)
        st = self.multigrid.hierarchy.backward(float(dt), start_level, grad_mask)
        self.last_stats = st
        if self._fas_config.report_norms and report_norms:
            h = st["history"]
            print(f"  Initial:   |r0|     = {h[0]:.2e}")
            for k in range(1, len(h)):
                print(f"  V-cycle {k - 1}: |r|/|r0| = {h[k] / h[0]:.2e}")
        return st
