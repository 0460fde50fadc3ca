"""Per-level forward and adjoint operators (mirror of glide/operators.py).

Every method launches the fused sm_100a kernels of libglide_b200.so through
the C ABI.  Differences from the reference's host code, by design:
  * a Vanka sweep is one fused kernel (grounding prologue, block solves, face
    averaging and the omega-update); the per-sweep `delta_*` buffers and the
    three axpys of glide/operators.py:243-251 do not exist;
  * residual norms are reduced on the device in a fixed order.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

from . import _lib


class _Synced:
    """Dataclass mixin: every public attribute write re-pushes the config."""

    def __setattr__(self, k, v):
        object.__setattr__(self, k, v)
        push = self.__dict__.get("_push")
        if push is not None and not k.startswith("_"):
            push()

    def _bind(self, push):
        object.__setattr__(self, "_push", push)


@dataclass
class NewtonConfig(_Synced):
    """Local Newton of the Vanka block solve (glide/operators.py:314-319).

    `relaxation` is kept for API parity; as in the reference kernel
    (glide/cuda/vanka.cu:615) the local update uses 0.5.
    """
    steps: int = 30
    relaxation: float = 0.5
    ssa_damping: float = 0.01
    mc_damping: float = 1.0


def _no_hook(i):
    return None


_no_hook._glide_default = True


@dataclass
class VankaConfig(_Synced):
    """Vanka smoother options (glide/operators.py:321-327).  A user
    `hook_func(i)` makes sweeps run one launch at a time with the hook
    called after each, as in the reference."""
    omega: float = 0.5
    newton_config: NewtonConfig = field(default_factory=NewtonConfig)
    relax_phi: float = 0.0
    hook_interval: int = 1
    hook_func: Callable[[int], None] = field(default_factory=lambda: _no_hook)


def _bind_vanka(cfg: VankaConfig, hier, adjoint: bool, level: int):
    def push():
        n = cfg.newton_config
        hier.set_vanka(adjoint, level, omega=cfg.omega, newton_steps=n.steps, relaxation=n.relaxation,
                       ssa_damping=n.ssa_damping, mc_damping=n.mc_damping, relax_phi=cfg.relax_phi)
    cfg._bind(push)
    cfg.newton_config._bind(push)
    push()


class ForwardOperators:
    """Residual, grounding and smoother of one level (glide/operators.py:10-312)."""

    def __init__(self, grid):
        self.grid = grid
        self._h = grid._hier
        self._l = grid.level
        self.vanka_config = VankaConfig()
        _bind_vanka(self.vanka_config, self._h, False, self._l)

    def _v(self, name):
        return self._h.view(name, self._l)

    r_u = property(lambda s: s._v("r_u"))
    r_v = property(lambda s: s._v("r_v"))
    r_H = property(lambda s: s._v("r_H"))
    f_u = property(lambda s: s._v("f_u"))
    f_v = property(lambda s: s._v("f_v"))
    f_H = property(lambda s: s._v("f_H"))
    F_u = property(lambda s: s._v("F_u"))
    F_v = property(lambda s: s._v("F_v"))
    F_H = property(lambda s: s._v("F_H"))
    gamma = property(lambda s: s._v("gamma"))
    var_u = property(lambda s: s._v("var_u"))
    var_v = property(lambda s: s._v("var_v"))
    var_H = property(lambda s: s._v("var_H"))
    jvp_u = property(lambda s: s._v("jvp_u"))
    jvp_v = property(lambda s: s._v("jvp_v"))
    jvp_H = property(lambda s: s._v("jvp_H"))

    def compute_jvp(self, dt, use_mask=True, freeze_calving=False, freeze_phi=False, return_norms=False):
        """jvp = J(x) var with the reference's row conventions
        (glide/operators.py:129-171); phi is recomputed first unless frozen.
        use_mask=False reads the mask as 0 and freeze_calving=True sets the
        calving rate to 0, as the reference does.  return_norms is accepted
        and, as in the reference, nothing is returned."""
        if not freeze_phi:
            self.compute_phi()
        flags = (_lib.USE_MASK if use_mask else 0) | (_lib.FREEZE_CALVING if freeze_calving else 0)
        self._h.jvp(self._l, dt, reference_rows=True, flags=flags)

    def compute_residual(self, dt, use_mask=True, operator_only=False, freeze_calving=False,
                         freeze_phi=False, return_norms=False):
        flags = ((_lib.USE_MASK if use_mask else 0) | (_lib.OPERATOR_ONLY if operator_only else 0) |
                 (_lib.FREEZE_CALVING if freeze_calving else 0) | (_lib.FREEZE_PHI if freeze_phi else 0))
        return self._h.residual(self._l, dt, flags, norms=return_norms)

    def compute_phi(self, relaxation=0.0):
        self._h.compute_phi(self._l, relaxation)

    def vanka_sweep(self, dt, n_iter, freeze_calving=False, freeze_phi=False, newton_iters=None):
        flags = (_lib.FREEZE_CALVING if freeze_calving else 0) | (_lib.FREEZE_PHI if freeze_phi else 0)
        hook = self.vanka_config.hook_func
        if getattr(hook, "_glide_default", False):
            self._h.vanka_sweep(self._l, dt, n_iter, flags, newton_iters)
            return
        for i in range(n_iter):  # a user hook runs between sweeps
            self._h.vanka_sweep(self._l, dt, 1, flags, newton_iters)
            hook(i)

    def vanka_dump(self, dt):
        """Local 5x5 Vanka matrices and residuals of every cell at the current
        state (glide/operators.py:253-273); returns new tensors J (ny*nx, 25)
        and r (ny*nx, 5)."""
        return self._h.vanka_dump(self._l, dt)

    def vanka_smooth(self, dt, freeze_calving=False, freeze_phi=False):
        """One smoother pass.  Unlike the reference, the update is applied in the
        same fused kernel (there are no separate delta buffers)."""
        self.vanka_sweep(dt, 1, freeze_calving=freeze_calving, freeze_phi=freeze_phi)

    def set_rhs(self, dt):
        self._h.set_rhs(self._l, dt)


class AdjointOperators:
    """Transpose residual, adjoint smoother and gradients (glide/operators.py:330-593)."""

    def __init__(self, grid):
        self.grid = grid
        self._h = grid._hier
        self._l = grid.level
        self.vanka_config = VankaConfig()
        _bind_vanka(self.vanka_config, self._h, True, self._l)

    def _v(self, name):
        return self._h.view(name, self._l)

    r_u = property(lambda s: s._v("adj_r_u"))
    r_v = property(lambda s: s._v("adj_r_v"))
    r_H = property(lambda s: s._v("adj_r_H"))
    f_u = property(lambda s: s._v("adj_f_u"))
    f_v = property(lambda s: s._v("adj_f_v"))
    f_H = property(lambda s: s._v("adj_f_H"))
    vjp_u = property(lambda s: s._v("vjp_u"))
    vjp_v = property(lambda s: s._v("vjp_v"))
    vjp_H = property(lambda s: s._v("vjp_H"))
    gamma = property(lambda s: s._v("gamma"))

    def compute_residual(self, dt, use_mask=True, freeze_calving=False, return_norms=False):
        return self._h.adjoint_residual(self._l, dt, norms=return_norms)

    def compute_vjp(self, dt, use_mask=True, use_forcing=False, freeze_calving=False):
        self._h.vjp(self._l, dt)

    def vanka_sweep(self, dt, n_iter, freeze_calving=False):
        self._h.adjoint_sweep(self._l, dt, n_iter)

    def vanka_smooth(self, dt, freeze_calving=False):
        """One adjoint smoother pass (glide/operators.py:474-515).  As in the
        forward operators, the update lambda -= omega * delta is applied in the
        same fused kernel (there are no separate delta buffers)."""
        self.vanka_sweep(dt, 1, freeze_calving=freeze_calving)

    def compute_gradient_beta(self):
        self._h.gradients(self._l, 1.0, _lib.GRAD_BETA)

    def compute_gradient_bed(self):
        self._h.gradients(self._l, 1.0, _lib.GRAD_BED)

    def compute_gradient_H_prev(self, dt):
        self._h.gradients(self._l, dt, _lib.GRAD_H_PREV)

    def compute_gradient_smb(self):
        self._h.gradients(self._l, 1.0, _lib.GRAD_SMB)
