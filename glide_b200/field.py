"""Fields, constants and option wrappers (mirror of glide/field.py).

A `Field` is a named array of one hierarchy level; its `.data` is a torch
tensor aliasing the device arena, so in-place writes (`f.data[:, :] = x`)
land directly in the solver's memory.  Restates the container semantics of
glide/field.py:41-112 and :212-286 (the xarray export of :115-210 is I/O and
not part of the solver path).
"""
from __future__ import annotations

from enum import Enum
from typing import Any, Callable

import torch


class GridEntity(str, Enum):
    CELL = "cell"
    VERTICAL_FACET = "vertical_facet"
    HORIZONTAL_FACET = "horizontal_facet"


class Field:
    def __init__(self, hier, name: str, level: int, grid_entity: GridEntity, dx: float, grid=None,
                 units: str | None = None, attrs: dict | None = None, grad_name: str | None = None):
        self._hier = hier
        self.name = name
        self.level = level
        self.grid_entity = grid_entity
        self.dx = dx
        self.grid = grid
        self.units = units
        self.attrs = attrs or {}
        self._grad_name = grad_name
        self._grad = None

    @property
    def data(self) -> torch.Tensor:
        return self._hier.view(self.name, self.level)

    @data.setter
    def data(self, value):
        self.set(value)

    def set(self, value) -> None:
        """Copy an array (any device/dtype) or fill a scalar (glide/field.py:52-56)."""
        self._hier.set(self.name, self.level, value, restrict_down=False)

    def zero(self) -> None:
        self.set(0.0)

    @property
    def grad(self) -> torch.Tensor:
        if self._grad_name is not None:
            return self._hier.view(self._grad_name, self.level)
        if self._grad is None:
            self._grad = torch.zeros_like(self.data)
        return self._grad

    def has_grad(self) -> bool:
        return self._grad_name is not None or self._grad is not None

    def zero_grad(self) -> None:
        if self._grad_name is not None:
            self._hier.set(self._grad_name, self.level, 0.0)
        elif self._grad is not None:
            self._grad.zero_()

    def to_cell(self) -> torch.Tensor:
        d = self.data
        if self.grid_entity is GridEntity.VERTICAL_FACET:
            return 0.5 * (d[:, 1:] + d[:, :-1])
        if self.grid_entity is GridEntity.HORIZONTAL_FACET:
            return 0.5 * (d[1:] + d[:-1])
        return d

    @property
    def compact_string(self):
        r, c = self.data.shape
        return f"Field: {self.name}, {self.units}, ({r}, {c})"

    def __repr__(self):
        d = self.data
        return f"Field: {self.name}\n{d}\n{tuple(d.shape)}, {d.dtype}, {self.units}"


class SubgridField(Field):
    quantiles: Any | None = None


class Constant:
    """A scalar parameter of one level; `set` pushes it to the solver."""

    def __init__(self, value, name: str | None = None, units: str | None = None,
                 attrs: dict | None = None, on_set: Callable[[float], None] | None = None):
        self.value = float(value)
        self.name = name
        self.units = units
        self.attrs = attrs or {}
        self._on_set = on_set
        self._grad = None

    def set(self, value) -> None:
        self.value = float(value)
        if self._on_set is not None:
            self._on_set(self.value)

    @property
    def grad(self):
        if self._grad is None:
            self._grad = 0.0
        return self._grad

    def has_grad(self) -> bool:
        return self._grad is not None

    def zero_grad(self) -> None:
        if self._grad is not None:
            self._grad = 0.0

    def __repr__(self):
        return f"Constant: {self.name}, {self.value:.3f}, {self.units}"


class LocalOption:
    """Getter/setter pair for one option of a single config (glide/field.py:254-267)."""

    def __init__(self, getter, setter, name: str):
        self._getter = getter
        self._setter = setter
        self._name = name

    def get(self):
        return self._getter()

    def set(self, value):
        self._setter(value)

    def __repr__(self):
        return f"{self._name}={self.get()!r}"


class BroadcastOption:
    """One option broadcast over every level's config (glide/field.py:270-286)."""

    def __init__(self, levels, getter, attr_name: str):
        self._levels = levels
        self._getter = getter
        self._attr_name = attr_name

    def get(self):
        return getattr(self._getter(self._levels[0]), self._attr_name)

    def set(self, value):
        for lev in self._levels:
            setattr(self._getter(lev), self._attr_name, value)

    def __repr__(self):
        return f"{self._attr_name}={self.get()!r}"
