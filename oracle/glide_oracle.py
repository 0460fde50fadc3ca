"""CPU oracle: NumPy sequencing over the C++ restated operators.

TEST INFRASTRUCTURE.  Only tests/, `__graft_entry__.smoke()` and the CPU
baseline leg of bench.py use this module; the product (glide_b200) never
imports it.

`OracleHierarchy` restates the reference's host-side sequencing in this
project's own code:
  set_rhs / vanka sweep                glide/operators.py:243-251, :275-276
  FASCD solve + V-cycle                glide/multigrid.py:502-645
  FASAdjoint solve + V-cycle           glide/multigrid.py:873-973
  hierarchy restriction of fields      glide/multigrid.py:54-116, :264-283
  backward (adjoint + gradients)       glide/model.py:74-94, glide/operators.py:526-593
and calls the C++ restatement of the kernels in libglide_oracle.so
(oracle/glide_oracle.cpp).  Arrays are contiguous NumPy arrays in binary64
(dtype=np.float64) or binary32.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = HERE / "libglide_oracle.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run python oracle/build_oracle.py")
        _LIB = ctypes.CDLL(str(path))
    return _LIB


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


# Default physical constants of a level (glide/grid.py:28-138).
PHYS_DEFAULTS = dict(n=3.0, eps_reg=1e-6, flotation_reg_driving=0.1, m=1.0, u_reg=1.0,
                     water_drag=1e-5, flotation_reg_sliding=0.1, calving_rate=0.0,
                     flotation_reg_calving=0.1, thklim=0.1)
PHYS_ORDER = ("n", "eps_reg", "flotation_reg_driving", "m", "u_reg", "water_drag",
              "flotation_reg_sliding", "calving_rate", "flotation_reg_calving")


@dataclass
class FASConfig:
    """Forward and adjoint schedule; defaults of glide/multigrid.py:672-682."""
    freeze_coarse_calving: bool = True
    freeze_coarse_phi: bool = True
    coarsest_steps: int = 200
    pre_steps: int = 10
    post_steps: int = 20
    finest_steps: int = 50
    maximum_vcycles: int = 10
    relative_tolerance: float = 1e-3
    absolute_tolerance: float = 5.0


@dataclass
class VankaCfg:
    """glide/operators.py:314-327 defaults."""
    omega: float = 0.5
    steps: int = 30
    ssa_damping: float = 0.01
    mc_damping: float = 1.0
    relax_phi: float = 0.0


class OracleLevel:
    def __init__(self, ny, nx, dx, dtype):
        self.ny, self.nx, self.dx, self.dtype = ny, nx, float(dx), dtype
        z = lambda *s: np.zeros(s, dtype)
        U, V, C = (ny, nx + 1), (ny + 1, nx), (ny, nx)
        self.u, self.v, self.H = z(*U), z(*V), z(*C)
        self.H_prev, self.phi, self.mask = z(*C), z(*C), z(*C)
        self.bed, self.B, self.beta, self.smb = z(*C), z(*C), z(*C), z(*C)
        self.f_u, self.f_v, self.f_H = z(*U), z(*V), z(*C)
        self.r_u, self.r_v, self.r_H = z(*U), z(*V), z(*C)
        self.F_u, self.F_v, self.F_H = z(*U), z(*V), z(*C)
        self.d_u, self.d_v, self.d_H = z(*U), z(*V), z(*C)
        self.gamma = z(*C)
        self.w_u, self.w_v, self.w_H = z(*U), z(*V), z(*C)
        self.y_u, self.y_v, self.y_H = z(*U), z(*V), z(*C)
        self.z_u, self.z_v, self.z_H = z(*U), z(*V), z(*C)
        self.chi, self.phi_s = z(*C), z(*C)
        # adjoint
        self.l_u, self.l_v, self.l_H = z(*U), z(*V), z(*C)
        self.af_u, self.af_v, self.af_H = z(*U), z(*V), z(*C)
        self.ar_u, self.ar_v, self.ar_H = z(*U), z(*V), z(*C)
        self.vjp_u, self.vjp_v, self.vjp_H = z(*U), z(*V), z(*C)
        self.dl_u, self.dl_v, self.dl_H = z(*U), z(*V), z(*C)
        self.wl_u, self.wl_v, self.wl_H = z(*U), z(*V), z(*C)
        self.zl_u, self.zl_v, self.zl_H = z(*U), z(*V), z(*C)
        self.g_beta, self.g_bed = z(*C), z(*C)
        self.phys = dict(PHYS_DEFAULTS)
        self.gamma.fill(self.phys["thklim"])
        self.vanka = VankaCfg()
        self.adj_vanka = VankaCfg()

    # -- kernel wrappers -------------------------------------------------
    @property
    def suf(self):
        return "f64" if self.dtype == np.float64 else "f32"

    def _phys(self, dt, calving_rate=None):
        vals = [self.phys[k] for k in PHYS_ORDER]
        if calving_rate is not None:
            vals[PHYS_ORDER.index("calving_rate")] = calving_rate
        vals += [self.dx, dt]
        return (ctypes.c_double * 11)(*vals)

    def _level_args(self, dt, f=None, calving_rate=None, state=None):
        f_u, f_v, f_H = f if f is not None else (self.f_u, self.f_v, self.f_H)
        u, v, H = state if state is not None else (self.u, self.v, self.H)
        return [ctypes.c_int(self.ny), ctypes.c_int(self.nx), _p(u), _p(v), _p(H),
                _p(self.phi), _p(self.mask), _p(f_u), _p(f_v), _p(f_H), _p(self.bed),
                _p(self.B), _p(self.beta), _p(self.gamma), self._phys(dt, calving_rate)]

    def compute_phi(self, relax=0.0):
        getattr(lib(), "go_grounded_" + self.suf)(
            ctypes.c_int(self.ny), ctypes.c_int(self.nx), _p(self.phi), _p(self.H), _p(self.bed),
            ctypes.c_double(self.phys["flotation_reg_driving"]), ctypes.c_double(relax))

    def residual(self, dt, use_mask=True, operator_only=False, freeze_calving=False,
                 freeze_phi=False):
        """ForwardOperators.compute_residual, glide/operators.py:71-127."""
        if not freeze_phi:
            self.compute_phi()
        out = (self.F_u, self.F_v, self.F_H) if operator_only else (self.r_u, self.r_v, self.r_H)
        cr = 0.0 if freeze_calving else None
        getattr(lib(), "go_residual_" + self.suf)(
            *self._level_args(dt, calving_rate=cr), ctypes.c_int(0 if operator_only else 1),
            ctypes.c_int(1 if use_mask else 0), *[_p(a) for a in out])
        return out

    def norms(self, arrs):
        return tuple(float(np.sqrt(np.sum(a.astype(np.float64) ** 2))) for a in arrs)

    def vanka_sweep(self, dt, n, freeze_calving=False, freeze_phi=False, iters=None):
        """ForwardOperators.vanka_sweep, glide/operators.py:194-251."""
        cfg = self.vanka
        cr = 0.0 if freeze_calving else None
        for _ in range(n):
            if not freeze_phi:
                self.compute_phi(cfg.relax_phi)
            it = np.zeros((self.ny, self.nx), np.int32) if iters is not None else None
            getattr(lib(), "go_vanka_" + self.suf)(
                *self._level_args(dt, calving_rate=cr), ctypes.c_int(cfg.steps),
                ctypes.c_double(cfg.ssa_damping), ctypes.c_double(cfg.mc_damping),
                _p(self.d_u), _p(self.d_v), _p(self.d_H), _p(self.mask),
                _p(it) if it is not None else None)
            if iters is not None:
                iters.append(it)
            w = self.dtype(cfg.omega)
            self.u += w * self.d_u
            self.v += w * self.d_v
            self.H += w * self.d_H

    def vanka_dump(self, dt):
        """ForwardOperators.vanka_dump, glide/operators.py:253-273: the local
        5x5 systems of every cell at the current state and phi."""
        J = np.zeros((self.ny * self.nx, 25), self.dtype)
        r = np.zeros((self.ny * self.nx, 5), self.dtype)
        getattr(lib(), "go_vanka_dump_" + self.suf)(*self._level_args(dt), _p(J), _p(r))
        return J, r

    def vjp(self, dt, lam, use_forcing, out, f=None):
        getattr(lib(), "go_vjp_" + self.suf)(
            *self._level_args(dt, f=f), *[_p(a) for a in lam], ctypes.c_int(1 if use_forcing else 0),
            *[_p(a) for a in out])

    def adj_residual(self, dt):
        """AdjointOperators.compute_residual, glide/operators.py:379-425."""
        for a in (self.ar_u, self.ar_v, self.ar_H):
            a.fill(0)
        self.vjp(dt, (self.l_u, self.l_v, self.l_H), True, (self.ar_u, self.ar_v, self.ar_H),
                 f=(self.af_u, self.af_v, self.af_H))
        return self.ar_u, self.ar_v, self.ar_H

    def adj_vjp(self, dt):
        self.vjp(dt, (self.l_u, self.l_v, self.l_H), False, (self.vjp_u, self.vjp_v, self.vjp_H),
                 f=(self.af_u, self.af_v, self.af_H))

    def adj_sweep(self, dt, n):
        """AdjointOperators.vanka_sweep, glide/operators.py:517-524."""
        cfg = self.adj_vanka
        for _ in range(n):
            self.adj_residual(dt)
            getattr(lib(), "go_vanka_adjoint_" + self.suf)(
                *self._level_args(dt), ctypes.c_double(cfg.ssa_damping),
                ctypes.c_double(cfg.mc_damping), _p(self.ar_u), _p(self.ar_v), _p(self.ar_H),
                _p(self.dl_u), _p(self.dl_v), _p(self.dl_H))
            w = self.dtype(cfg.omega)
            self.l_u -= w * self.dl_u
            self.l_v -= w * self.dl_v
            self.l_H -= w * self.dl_H

    def gradients(self):
        getattr(lib(), "go_gradients_" + self.suf)(
            *self._level_args(0.0), _p(self.l_u), _p(self.l_v), _p(self.g_beta), _p(self.g_bed))


def _restrict_u(f, c):
    getattr(lib(), "go_restrict_u_" + _suf(f))(_p(f), _p(c), c.shape[0], c.shape[1] - 1)


def _restrict_v(f, c):
    getattr(lib(), "go_restrict_v_" + _suf(f))(_p(f), _p(c), c.shape[0] - 1, c.shape[1])


def _restrict_cell(f, c, how="avg"):
    code = {"avg": 0, "max": 1, "min": 2, "var": 3}[how]
    getattr(lib(), "go_restrict_cell_" + _suf(f))(_p(f), _p(c), c.shape[0], c.shape[1], code)


def _prolong_u(c, f, bilinear=True):
    getattr(lib(), "go_prolong_u_" + _suf(f))(_p(c), _p(f), f.shape[0], f.shape[1] - 1, int(bilinear))


def _prolong_v_as_reference(c, f, bilinear=True):
    # The reference prolongates v-face data with its u-face kernel, handing it
    # the v arrays' memory and the sizes (2*(nyc), 2*nxc) derived from the v
    # shapes (glide/multigrid.py:212-235).  Reproduced on the same memory.
    nyc = c.shape[0] - 1
    getattr(lib(), "go_prolong_u_" + _suf(f))(_p(c), _p(f), 2 * nyc, 2 * c.shape[1], int(bilinear))


def _prolong_v(c, f, bilinear=True):
    getattr(lib(), "go_prolong_v_" + _suf(f))(_p(c), _p(f), f.shape[0] - 1, f.shape[1], int(bilinear))


def _prolong_cell(c, f, bilinear=False):
    getattr(lib(), "go_prolong_cell_" + _suf(f))(_p(c), _p(f), f.shape[0], f.shape[1], int(bilinear))


def _suf(a):
    return "f64" if a.dtype == np.float64 else "f32"


class OracleHierarchy:
    """Level hierarchy plus the forward (FASCD) and adjoint solvers."""

    def __init__(self, ny, nx, dx, n_levels, dtype=np.float64, reference_quirks=True):
        self.dtype = dtype
        self.levels = [OracleLevel(ny, nx, dx, dtype)]
        for _ in range(1, n_levels):
            f = self.levels[-1]
            self.levels.append(OracleLevel(f.ny // 2, f.nx // 2, f.dx * 2, dtype))
        self.fas = FASConfig()
        self.adj = FASConfig()
        self.quirks = reference_quirks
        self.history = []

    # -- hierarchy field setting (HierarchyFieldManager.set) ----------------
    def set_field(self, name, value, start_level=0):
        lv = self.levels
        arr = getattr(lv[start_level], name)
        arr[...] = np.asarray(value, dtype=self.dtype)
        how = "max" if name == "mask" else "avg"
        for l in range(start_level, len(lv) - 1):
            f, c = getattr(lv[l], name), getattr(lv[l + 1], name)
            if name in ("u", "l_u"):
                _restrict_u(f, c)
            elif name in ("v", "l_v"):
                _restrict_v(f, c)
            else:
                _restrict_cell(f, c, how)

    def set_phys(self, **kw):
        for lev in self.levels:
            for k, v in kw.items():
                lev.phys[k] = float(v)
            lev.gamma.fill(lev.phys["thklim"])

    def restrict_state(self, f, c):
        _restrict_u(f.u, c.u)
        _restrict_v(f.v, c.v)
        _restrict_cell(f.H, c.H)
        _restrict_cell(f.H_prev, c.H_prev)
        _restrict_cell(f.phi, c.phi)
        _restrict_cell(f.mask, c.mask, "max")

    def _prolong_v(self, c, f):
        if self.quirks:
            _prolong_v_as_reference(c, f)
        else:
            _prolong_v(c, f)

    # -- forward -----------------------------------------------------------
    def solve(self, dt, start_level=0):
        """FASCDSolver.solve, glide/multigrid.py:502-533."""
        self.dt = dt
        top = self.levels[start_level]
        top.f_H[...] = top.H_prev / self.dtype(dt) + top.smb
        r0 = np.sqrt(sum(x ** 2 for x in top.norms(top.residual(dt))))
        self.history = [r0]
        rel, ab, it = 1.0, r0, 0
        cfg = self.fas
        while rel > cfg.relative_tolerance and ab > cfg.absolute_tolerance and it < cfg.maximum_vcycles:
            self.vcycle(start_level, finest=True)
            ab = np.sqrt(sum(x ** 2 for x in top.norms(top.residual(dt, freeze_phi=True))))
            rel = ab / r0
            self.history.append(ab)
            it += 1
        return it

    def _sweep(self, lev, n, coarse, gamma=None):
        cfg = self.fas
        if gamma is not None:
            lev.gamma[...] = gamma
        lev.vanka_sweep(self.dt, n, freeze_calving=coarse and cfg.freeze_coarse_calving,
                        freeze_phi=coarse and cfg.freeze_coarse_phi)
        lev.gamma.fill(lev.phys["thklim"])

    def vcycle(self, l, finest=False):
        """FASCDSolver.vcycle, glide/multigrid.py:536-645."""
        coarse = not finest
        cfg = self.fas
        dt = self.dt
        lev = self.levels[l]
        if finest:
            lev.w_u[...] = lev.u
            lev.w_v[...] = lev.v
            lev.w_H[...] = lev.H
            lev.chi[...] = self.dtype(lev.phys["thklim"]) - lev.H
        if l == len(self.levels) - 1:
            self._sweep(lev, cfg.coarsest_steps, coarse, lev.w_H + lev.chi)
            return
        nxt = self.levels[l + 1]
        _restrict_cell(lev.chi, nxt.chi, "max")
        _prolong_cell(-nxt.chi, lev.phi_s, bilinear=False)
        lev.phi_s += lev.chi
        self._sweep(lev, cfg.pre_steps, coarse, lev.w_H + lev.phi_s)
        lev.y_u[...] = lev.u - lev.w_u
        lev.y_v[...] = lev.v - lev.w_v
        lev.y_H[...] = lev.H - lev.w_H
        self.restrict_state(lev, nxt)
        nxt.w_u[...] = nxt.u
        nxt.w_v[...] = nxt.v
        nxt.w_H[...] = nxt.H
        lev.residual(dt, use_mask=False, freeze_calving=coarse and cfg.freeze_coarse_calving,
                     freeze_phi=True)
        _restrict_u(lev.r_u, nxt.r_u)
        _restrict_v(lev.r_v, nxt.r_v)
        _restrict_cell(lev.r_H, nxt.r_H)
        nxt.residual(dt, use_mask=False, operator_only=True,
                     freeze_calving=cfg.freeze_coarse_calving, freeze_phi=cfg.freeze_coarse_phi)
        nxt.f_u[...] = nxt.F_u - nxt.r_u
        nxt.f_v[...] = nxt.F_v - nxt.r_v
        nxt.f_H[...] = nxt.F_H - nxt.r_H
        self.vcycle(l + 1)
        nxt.z_u[...] = nxt.u - nxt.w_u
        nxt.z_v[...] = nxt.v - nxt.w_v
        nxt.z_H[...] = nxt.H - nxt.w_H
        _prolong_u(nxt.z_u, lev.z_u)
        self._prolong_v(nxt.z_v, lev.z_v)
        _prolong_cell(nxt.z_H, lev.z_H, bilinear=False)
        lev.z_u += lev.y_u
        lev.z_v += lev.y_v
        lev.z_H += lev.y_H
        lev.u[...] = lev.w_u + lev.z_u
        lev.v[...] = lev.w_v + lev.z_v
        lev.H[...] = lev.w_H + lev.z_H
        self._sweep(lev, cfg.post_steps, coarse, lev.w_H + lev.chi)
        if finest:
            lev.vanka_sweep(dt, cfg.finest_steps, freeze_phi=False, freeze_calving=False)

    # -- adjoint -----------------------------------------------------------
    def adjoint_solve(self, dt, start_level=0):
        """FASAdjointSolver.solve, glide/multigrid.py:873-903."""
        self.dt = dt
        top = self.levels[start_level]
        r0 = np.sqrt(sum(x ** 2 for x in top.norms(top.adj_residual(dt))))
        self.adj_history = [r0]
        rel, ab, it = 1.0, r0, 0
        cfg = self.adj
        while rel > cfg.relative_tolerance and ab > cfg.absolute_tolerance and it < cfg.maximum_vcycles:
            self.adj_vcycle(start_level, finest=True)
            ab = np.sqrt(sum(x ** 2 for x in top.norms(top.adj_residual(dt))))
            rel = ab / r0
            self.adj_history.append(ab)
            it += 1
        return it

    def adj_vcycle(self, l, finest=False):
        """FASAdjointSolver.vcycle, glide/multigrid.py:905-973."""
        cfg = self.adj
        dt = self.dt
        lev = self.levels[l]
        if l == len(self.levels) - 1:
            lev.adj_sweep(dt, cfg.coarsest_steps)
            return
        nxt = self.levels[l + 1]
        lev.adj_sweep(dt, cfg.pre_steps)
        self.restrict_state(lev, nxt)
        _restrict_u(lev.l_u, nxt.l_u)
        _restrict_v(lev.l_v, nxt.l_v)
        _restrict_cell(lev.l_H, nxt.l_H)
        nxt.wl_u[...] = nxt.l_u
        nxt.wl_v[...] = nxt.l_v
        nxt.wl_H[...] = nxt.l_H
        lev.adj_residual(dt)
        _restrict_u(lev.ar_u, nxt.ar_u)
        _restrict_v(lev.ar_v, nxt.ar_v)
        _restrict_cell(lev.ar_H, nxt.ar_H)
        nxt.vjp_u.fill(0); nxt.vjp_v.fill(0); nxt.vjp_H.fill(0)
        nxt.adj_vjp(dt)
        nxt.af_u[...] = nxt.vjp_u - nxt.ar_u
        nxt.af_v[...] = nxt.vjp_v - nxt.ar_v
        nxt.af_H[...] = nxt.vjp_H - nxt.ar_H
        self.adj_vcycle(l + 1)
        nxt.zl_u[...] = nxt.l_u - nxt.wl_u
        nxt.zl_v[...] = nxt.l_v - nxt.wl_v
        nxt.zl_H[...] = nxt.l_H - nxt.wl_H
        _prolong_u(nxt.zl_u, lev.zl_u)
        self._prolong_v(nxt.zl_v, lev.zl_v)
        _prolong_cell(nxt.zl_H, lev.zl_H, bilinear=True)
        lev.l_u += lev.zl_u
        lev.l_v += lev.zl_v
        lev.l_H += lev.zl_H
        lev.adj_sweep(dt, cfg.post_steps)
        if finest:
            lev.adj_sweep(dt, cfg.finest_steps)

    def backward(self, dt, dJdu=None, dJdv=None, dJdH=None, start_level=0):
        """IceDynamics.backward, glide/model.py:74-94."""
        top = self.levels[start_level]
        for arr, g in ((top.af_u, dJdu), (top.af_v, dJdv), (top.af_H, dJdH)):
            if g is None:
                arr.fill(0)
            else:
                arr[...] = -np.asarray(g, dtype=self.dtype)
        self.adjoint_solve(dt, start_level)
        top.gradients()
        g_H_prev = -top.l_H / self.dtype(dt)
        g_smb = -top.l_H.copy()
        return dict(beta=top.g_beta.copy(), bed=top.g_bed.copy(), H_prev=g_H_prev, smb=g_smb)
