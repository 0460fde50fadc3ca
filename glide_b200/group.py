"""Grouped solves: one solve of many hierarchies in grouped launches.

`HierarchyGroup` wraps glide_group_* (include/glide_b200.h).  Each kind of
launch of a V-cycle is issued once for all members, its blocks mapped to
(member, tile); the whole cycle of every member is one CUDA graph, and each
member's convergence test runs on the device.  A member computes exactly what
its own `Hierarchy.forward` / `backward` computes.

No counterpart in the reference, which solves one grid at a time
(IceDynamics.forward / backward, glide/model.py:62-94).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .hierarchy import Hierarchy, _stream_ptr


class HierarchyGroup:
    """A fixed set of hierarchies of one precision ("fp64" or "fp32"), solved
    together.  The hierarchies stay usable on their own; they must not be
    driven from another thread while a group call runs."""

    def __init__(self, hierarchies: list[Hierarchy]):
        self.hierarchies = list(hierarchies)  # the group borrows their handles
        n = len(self.hierarchies)
        arr = (ctypes.c_void_p * n)(*[h.handle for h in self.hierarchies])
        out = ctypes.c_void_p()
        _lib.check(_lib.load().glide_group_create(arr, n, ctypes.byref(out)))
        self._g = out

    def __len__(self) -> int:
        return len(self.hierarchies)

    def close(self):
        g = getattr(self, "_g", None)
        if g is not None and g.value:
            try:
                torch.cuda.synchronize()
                _lib.load().glide_group_destroy(g)
            except Exception:
                pass
        self._g = None

    def __del__(self):
        self.close()

    def _stats(self):
        return (_lib.Stats * len(self.hierarchies))()

    def forward(self, dt: float, start_level: int = 0) -> list[dict]:
        """FASCD forward solve of every member (each with its own schedule,
        tolerances and cycle cap); the members' statistics in order."""
        st = self._stats()
        _lib.check(_lib.load().glide_group_forward(self._g, float(dt), int(start_level), st, _stream_ptr()))
        return [s.to_dict() for s in st]

    def backward(self, dt: float, start_level: int = 0, mask: int = _lib.GRAD_ALL) -> list[dict]:
        """Adjoint solve and gradients of every member (the right-hand sides
        and the start of lambda set on each member beforehand)."""
        st = self._stats()
        _lib.check(_lib.load().glide_group_backward(self._g, float(dt), int(start_level), int(mask), st,
                                                    _stream_ptr()))
        return [s.to_dict() for s in st]

    def set_tuning(self, waves: int | None = None, spoil_maps: bool | None = None):
        """Launch shape of the grouped launches: 0 (default) launches one
        block per tile; `waves` > 0 launches that many waves of the GPU's
        resident blocks, each block striding over the tiles.  `spoil_maps`
        uploads the staging maps without the tag the kernels check before
        their first copy (a test of that check: the next call fails with
        GLIDE_ERR_STATE)."""
        if waves is not None:
            _lib.check(_lib.load().glide_group_set_tuning(self._g, _lib.GROUP_TUNE_WAVES, int(waves)))
        if spoil_maps is not None:
            _lib.check(_lib.load().glide_group_set_tuning(self._g, _lib.GROUP_TUNE_SPOIL_MAPS, 1 if spoil_maps else 0))

    def counters(self) -> dict:
        """Grouped launches issued so far, and the shape of the last forward
        and adjoint cycles: grouped launches and the members' launches they
        carry."""
        n = ctypes.c_longlong()
        shape = (ctypes.c_int * 4)()
        _lib.check(_lib.load().glide_group_counters(self._g, ctypes.byref(n), shape))
        return {"launches": n.value, "forward_cycle": (shape[0], shape[1]), "adjoint_cycle": (shape[2], shape[3])}
