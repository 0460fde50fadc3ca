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
from .hierarchy import Hierarchy, transfer
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

    # ------------------------------------------------- level construction
    def create_grid_hierarchy(self, n_levels, restrict_fields=True):
        """glide/multigrid.py:54-60.  The device arena is sized for
        `self.n_levels` levels when the Multigrid is built, so the call
        re-derives the existing levels (restricting every field down from the
        finest when restrict_fields) and n_levels must equal that count."""
        if int(n_levels) != self.n_levels:
            raise ValueError(f"this Multigrid holds {self.n_levels} levels, fixed when it was built; "
                             f"build a new Multigrid for {n_levels}")
        levels = [self.finest_grid]
        for _ in range(1, self.n_levels):
            levels.append(self.create_coarse_grid(levels[-1], restrict_fields=restrict_fields))
        return self.levels

    def create_coarse_grid(self, parent_grid, restrict_fields=True):
        """glide/multigrid.py:62-79: the grid of half the cells and twice the
        spacing under `parent_grid`, its origin shifted by half a fine cell.
        A level of this hierarchy returns its existing child; any other grid
        (or the coarsest level) gets a new stand-alone Grid.  With
        restrict_fields, the state, geometry, rheology, sliding, calving and
        forcing are restricted into it."""
        child = parent_grid.child
        if child is None:
            child = Grid(parent_grid.ny // 2, parent_grid.nx // 2, parent_grid.dx * 2,
                         x0=parent_grid.x0 + parent_grid.dx / 2, y0=parent_grid.y0 - parent_grid.dx / 2,
                         crs=parent_grid.crs, parent=parent_grid, dtype=parent_grid._hier.dtype)
            parent_grid.child = child
        if restrict_fields:
            self.restrict_state(parent_grid, child)
            self.restrict_geometry(parent_grid, child)
            self.restrict_rheology(parent_grid, child)
            self.restrict_sliding(parent_grid, child)
            self.restrict_calving(parent_grid, child)
            self.restrict_forcing(parent_grid, child)
        return child

    # ------------------------------------------- grid-to-grid restriction
    def restrict_state(self, fine_grid, coarse_grid):
        """glide/multigrid.py:81-87."""
        f, c = fine_grid.state, coarse_grid.state
        self.restrict_vfacet(f.u.data, c.u.data)
        self.restrict_hfacet(f.v.data, c.v.data)
        self.restrict_cell(f.H.data, c.H.data)
        self.restrict_cell(f.H_prev.data, c.H_prev.data)
        self.restrict_cell(f.phi.data, c.phi.data)
        self.restrict_cell(f.mask.data, c.mask.data, method="max")

    def restrict_geometry(self, fine_grid, coarse_grid):
        """glide/multigrid.py:89-92."""
        self.restrict_cell(fine_grid.geometry.bed.data, coarse_grid.geometry.bed.data)
        coarse_grid.geometry.thklim.set(fine_grid.geometry.thklim.value)
        coarse_grid.geometry.flotation_reg_driving.set(fine_grid.geometry.flotation_reg_driving.value)

    def restrict_rheology(self, fine_grid, coarse_grid):
        """glide/multigrid.py:94-97."""
        self.restrict_cell(fine_grid.rheology.B.data, coarse_grid.rheology.B.data)
        coarse_grid.rheology.n.set(fine_grid.rheology.n.value)
        coarse_grid.rheology.eps_reg.set(fine_grid.rheology.eps_reg.value)

    def restrict_sliding(self, fine_grid, coarse_grid):
        """glide/multigrid.py:99-104."""
        self.restrict_cell(fine_grid.sliding.beta.data, coarse_grid.sliding.beta.data)
        for k in ("m", "u_reg", "water_drag", "flotation_reg_sliding"):
            getattr(coarse_grid.sliding, k).set(getattr(fine_grid.sliding, k).value)

    def restrict_calving(self, fine_grid, coarse_grid):
        """glide/multigrid.py:106-108."""
        coarse_grid.calving.calving_rate.set(fine_grid.calving.calving_rate.value)
        coarse_grid.calving.flotation_reg_calving.set(fine_grid.calving.flotation_reg_calving.value)

    def restrict_forcing(self, fine_grid, coarse_grid):
        """glide/multigrid.py:110-111."""
        self.restrict_cell(fine_grid.forcing.smb.data, coarse_grid.forcing.smb.data)

    def restrict_residual(self, fine_grid, coarse_grid):
        """glide/multigrid.py:113-116."""
        f, c = fine_grid.forward_operators, coarse_grid.forward_operators
        self.restrict_vfacet(f.r_u, c.r_u)
        self.restrict_hfacet(f.r_v, c.r_v)
        self.restrict_cell(f.r_H, c.r_H)

    # ------------------------------------------------ one-field transfers
    # glide/multigrid.py:118-259 over the kernels of glide/cuda/transfer.cu.
    # Arrays are 2-D CUDA tensors (float64 or float32); a missing output is
    # allocated with the input's dtype.  Fine cell counts must be even.
    def restrict_vfacet(self, fine_field, coarse_field=None):
        """u faces (ny, nx+1) -> (ny/2, nx/2+1): mean of the two fine faces on
        each coarse face."""
        ny, nx = fine_field.shape[0], fine_field.shape[1] - 1
        if coarse_field is None:
            coarse_field = fine_field.new_empty((ny // 2, nx // 2 + 1))
        _check_shape(coarse_field, (ny // 2, nx // 2 + 1))
        transfer("restrict_vfacet", fine_field, coarse_field, ny, nx)
        return coarse_field

    def restrict_hfacet(self, fine_field, coarse_field=None):
        """v faces (ny+1, nx) -> (ny/2+1, nx/2)."""
        ny, nx = fine_field.shape[0] - 1, fine_field.shape[1]
        if coarse_field is None:
            coarse_field = fine_field.new_empty((ny // 2 + 1, nx // 2))
        _check_shape(coarse_field, (ny // 2 + 1, nx // 2))
        transfer("restrict_hfacet", fine_field, coarse_field, ny, nx)
        return coarse_field

    def restrict_cell(self, fine_field, coarse_field=None, method="avg"):
        """Cells (ny, nx) -> (ny/2, nx/2): 2x2 mean, maximum, minimum or
        (population) variance."""
        if method not in ("avg", "max", "min", "var"):
            raise TypeError("Valid restriction methods: [avg,max,min]")
        ny, nx = fine_field.shape
        if coarse_field is None:
            coarse_field = fine_field.new_empty((ny // 2, nx // 2))
        _check_shape(coarse_field, (ny // 2, nx // 2))
        transfer("restrict_cell_" + method, fine_field, coarse_field, ny, nx)
        return coarse_field

    def prolongate_vfacet(self, coarse_field, fine_field=None, method="injection"):
        """u faces (nyc, nxc+1) -> (2 nyc, 2 nxc+1)."""
        if method not in ("injection", "bilinear"):
            raise TypeError("Valid prolongation methods: [injection, bilinear]")
        nyf, nxf = 2 * coarse_field.shape[0], 2 * (coarse_field.shape[1] - 1)
        if fine_field is None:
            fine_field = coarse_field.new_empty((nyf, nxf + 1))
        _check_shape(fine_field, (nyf, nxf + 1))
        transfer("prolongate_vfacet_" + method, coarse_field, fine_field, nyf, nxf)
        return fine_field

    def prolongate_hfacet(self, coarse_field, fine_field=None, method="injection"):
        """v faces (nyc+1, nxc) -> (2 nyc+1, 2 nxc).  With reference quirks on
        (the default) this runs what the reference runs: its u-face kernels
        over the v arrays' memory (square grids only); with them off, the
        v-face formulas."""
        if method not in ("injection", "bilinear"):
            raise TypeError("Valid prolongation methods: [injection, bilinear]")
        nyf, nxf = 2 * (coarse_field.shape[0] - 1), 2 * coarse_field.shape[1]
        if fine_field is None:
            fine_field = coarse_field.new_empty((nyf + 1, nxf))
        _check_shape(fine_field, (nyf + 1, nxf))
        op = ("prolongate_hfacet_as_vfacet_" if self.hierarchy.reference_quirks else "prolongate_hfacet_") + method
        transfer(op, coarse_field, fine_field, nyf, nxf)
        return fine_field

    def prolongate_cell(self, coarse_field, fine_field=None, method="injection"):
        """Cells (nyc, nxc) -> (2 nyc, 2 nxc)."""
        if method not in ("injection", "bilinear"):
            raise TypeError("Valid prolongation methods: [injection, bilinear]")
        nyf, nxf = 2 * coarse_field.shape[0], 2 * coarse_field.shape[1]
        if fine_field is None:
            fine_field = coarse_field.new_empty((nyf, nxf))
        _check_shape(fine_field, (nyf, nxf))
        transfer("prolongate_cell_" + method, coarse_field, fine_field, nyf, nxf)
        return fine_field


def _check_shape(t, shape):
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"expected an array of shape {tuple(shape)}, got {tuple(t.shape)}")


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

    def vcycle(self, l, finest=False):
        """One FASCD V-cycle from level l (glide/multigrid.py:536-645) with the
        dt of the last `solve` (or the dt attribute set by the caller); the
        right-hand side of level l must be set (ForwardOperators.set_rhs)."""
        if self.dt is None:
            raise AttributeError("dt is unset: call solve() first or set solver.dt")
        self.multigrid.hierarchy.vcycle(False, l, finest, self.dt)


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

    def vcycle(self, l, finest=False):
        """One linear FAS V-cycle of the adjoint system from level l
        (glide/multigrid.py:905-973) with the dt of the last `solve` (or the dt
        attribute set by the caller); the adjoint right-hand side of level l
        must be set."""
        if self.dt is None:
            raise AttributeError("dt is unset: call solve() first or set solver.dt")
        self.multigrid.hierarchy.vcycle(True, l, finest, self.dt)
