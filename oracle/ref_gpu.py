"""The reference's own CUDA kernels on the GPU, driven by a restatement of the
reference's host sequence (test infrastructure: a baseline timed beside the
product, never the product).

oracle/_ref/libglide_ref_gpu.so is the reference's glide/cuda/*.cu compiled
unmodified for sm_100a with --use_fast_math (oracle/build_oracle.py,
oracle/ref_gpu.cu).  The reference itself drives those kernels through CuPy,
which is not installable here, from Python that does not travel with this
repository; this module restates that host sequence on torch float32 device
arrays, one library call per CuPy call:

  ForwardOperators.compute_phi / set_rhs / compute_residual / vanka_smooth /
  vanka_sweep                         glide/operators.py:71-127, :173-251, :275
  AdjointOperators.compute_residual / compute_vjp / vanka_smooth /
  vanka_sweep / compute_gradient_*    glide/operators.py:379-600
  Multigrid.restrict_* / prolongate_* glide/multigrid.py:81-259 (prolongate_hfacet
                                      runs the u-face kernels, as there)
  FASCDSolver.solve / vcycle          glide/multigrid.py:502-645
  FASAdjointSolver.solve / vcycle     glide/multigrid.py:873-973
  IceDynamics.forward / backward      glide/model.py:65-94

with the kernels' launch geometry (16 x 16 blocks, stride 14, halo 1; 256
threads for transfers), binary32 scalars, element-wise updates as the
reference writes them (temporaries included) and norms by torch.linalg.norm
in place of cp.linalg.norm.  The grid must be square (the reference's
v-face prolongation runs the u-face kernels on v arrays).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libglide_ref_gpu.so"

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} was not built (the reference checkout was absent at build time)")
        _lib = ctypes.CDLL(str(LIB_PATH))
    return _lib


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _f(x):
    return ctypes.c_float(float(x))


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference kernel launch {what} failed: CUDA error {rc}")


STRIDE, HALO, BLOCK = 14, 1, 16
PHYS_ORDER = ("n", "eps_reg", "flotation_reg_driving", "m", "u_reg", "water_drag", "flotation_reg_sliding",
              "calving_rate", "flotation_reg_calving")
# glide/grid.py:28-138 defaults
PHYS_DEFAULTS = dict(n=3.0, eps_reg=1e-6, flotation_reg_driving=0.1, m=1.0, u_reg=1.0, water_drag=1e-5,
                     flotation_reg_sliding=0.1, calving_rate=0.0, flotation_reg_calving=0.1, thklim=0.1)
TRANSFER = {"restrict_vfacet": 0, "restrict_hfacet": 1, "restrict_cell_avg": 2, "restrict_cell_max": 3,
            "prolongate_vfacet_injection": 4, "prolongate_vfacet_bilinear": 5, "prolongate_cell_injection": 6,
            "prolongate_cell_bilinear": 7}


@dataclass
class FASConfig:
    """FASCDConfig / FASAdjointConfig defaults, glide/multigrid.py:672-682, :993-1001."""
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
class VankaConfig:
    """VankaConfig / NewtonConfig defaults, glide/operators.py:315-327."""
    omega: float = 0.5
    steps: int = 30
    relaxation: float = 0.5
    ssa_damping: float = 0.01
    mc_damping: float = 1.0
    relax_phi: float = 0.0


class RefLevel:
    """One grid level: its state, parameters, operator work arrays and the
    solvers' scratch, as binary32 device arrays."""

    def __init__(self, ny, nx, dx, device):
        self.ny, self.nx, self.dx = ny, nx, float(dx)
        z = lambda *s: torch.zeros(s, dtype=torch.float32, device=device)
        U, V, C = (ny, nx + 1), (ny + 1, nx), (ny, nx)
        for names, shape in ((("u", "f_u", "r_u", "F_u", "d_u", "w_u", "y_u", "z_u", "l_u", "af_u", "ar_u",
                                "vjp_u", "dl_u", "wl_u", "zl_u"), U),
                             (("v", "f_v", "r_v", "F_v", "d_v", "w_v", "y_v", "z_v", "l_v", "af_v", "ar_v",
                                "vjp_v", "dl_v", "wl_v", "zl_v"), V),
                             (("H", "H_prev", "phi", "mask", "bed", "B", "beta", "smb", "f_H", "r_H", "F_H",
                               "d_H", "w_H", "y_H", "z_H", "chi", "phi_s", "gamma", "l_H", "af_H", "ar_H",
                               "vjp_H", "dl_H", "wl_H", "zl_H", "g_beta", "g_bed"), C)):
            for n in names:
                setattr(self, n, z(*shape))
        self.phys = dict(PHYS_DEFAULTS)
        self.gamma.fill_(self.phys["thklim"])
        self.vanka = VankaConfig()
        self.adj_vanka = VankaConfig()
        self.grid = (nx // STRIDE + 1, ny // STRIDE + 1)

    def _phys(self, dt, calving_rate=None):
        vals = [self.phys[k] for k in PHYS_ORDER]
        if calving_rate is not None:
            vals[PHYS_ORDER.index("calving_rate")] = calving_rate
        return [_f(x) for x in (*vals, self.dx, dt)]

    def _geom(self):
        return (self.grid[0], self.grid[1], BLOCK, BLOCK)

    def _tail(self):
        return (self.ny, self.nx, STRIDE, HALO)

    def compute_phi(self, relax=0.0, stream=None):
        _check(lib().grg_compute_grounded(*self._geom(), _p(self.phi), _p(self.H), _p(self.bed),
                                          _f(self.phys["flotation_reg_driving"]), _f(relax), *self._tail(),
                                          stream), "compute_grounded")

    def set_rhs(self, dt):
        self.f_H[:, :] = self.H_prev / dt + self.smb

    def residual(self, dt, use_mask=True, operator_only=False, freeze_calving=False, freeze_phi=False,
                 norms=False, stream=None):
        if not freeze_phi:
            self.compute_phi(stream=stream)
        out = (self.F_u, self.F_v, self.F_H) if operator_only else (self.r_u, self.r_v, self.r_H)
        cr = 0.0 if freeze_calving else None
        _check(lib().grg_compute_residual(
            *self._geom(), *[_p(a) for a in out], _p(self.u), _p(self.v), _p(self.H), _p(self.phi),
            _p(self.mask), _p(self.f_u), _p(self.f_v), _p(self.f_H), _p(self.bed), _p(self.B), _p(self.beta),
            _p(self.gamma), int(not operator_only), int(use_mask), *self._phys(dt, cr), *self._tail(), stream),
            "compute_residual")
        if norms:
            return tuple(torch.linalg.norm(a) for a in out)

    def vanka_smooth(self, dt, freeze_calving=False, freeze_phi=False, stream=None):
        cfg = self.vanka
        if not freeze_phi:
            self.compute_phi(cfg.relax_phi, stream)
        for a in (self.d_u, self.d_v, self.d_H):
            a.fill_(0.0)
        cr = 0.0 if freeze_calving else None
        _check(lib().grg_vanka_smooth(
            *self._geom(), _p(self.d_u), _p(self.d_v), _p(self.d_H), _p(self.mask), _p(self.u), _p(self.v),
            _p(self.H), _p(self.phi), _p(self.f_u), _p(self.f_v), _p(self.f_H), _p(self.bed), _p(self.B),
            _p(self.beta), _p(self.gamma), *self._phys(dt, cr), *self._tail(), cfg.steps, _f(cfg.relaxation),
            _f(cfg.ssa_damping), _f(cfg.mc_damping), stream), "vanka_smooth")

    def vanka_sweep(self, dt, n, freeze_calving=False, freeze_phi=False, stream=None):
        w = torch.tensor(self.vanka.omega, dtype=torch.float32)
        for _ in range(n):
            self.vanka_smooth(dt, freeze_calving, freeze_phi, stream)
            self.u += w * self.d_u
            self.v += w * self.d_v
            self.H += w * self.d_H

    def _vjp(self, out, dt, use_forcing, stream):
        _check(lib().grg_compute_vjp(
            *self._geom(), *[_p(a) for a in out], _p(self.u), _p(self.v), _p(self.H), _p(self.l_u), _p(self.l_v),
            _p(self.l_H), _p(self.phi), _p(self.mask), _p(self.af_u), _p(self.af_v), _p(self.af_H), _p(self.bed),
            _p(self.B), _p(self.beta), _p(self.gamma), int(use_forcing), 1, *self._phys(dt), *self._tail(), stream),
            "compute_vjp")

    def adj_residual(self, dt, norms=False, stream=None):
        out = (self.ar_u, self.ar_v, self.ar_H)
        for a in out:
            a.fill_(0)
        self._vjp(out, dt, True, stream)
        if norms:
            return tuple(torch.linalg.norm(a) for a in out)

    def adj_vjp(self, dt, stream=None):
        out = (self.vjp_u, self.vjp_v, self.vjp_H)
        for a in out:
            a.fill_(0)
        self._vjp(out, dt, False, stream)

    def adj_sweep(self, dt, n, stream=None):
        cfg = self.adj_vanka
        w = torch.tensor(cfg.omega, dtype=torch.float32)
        for _ in range(n):
            self.adj_residual(dt, stream=stream)
            for a in (self.dl_u, self.dl_v, self.dl_H):
                a.fill_(0.0)
            _check(lib().grg_vanka_smooth_adjoint(
                *self._geom(), _p(self.dl_u), _p(self.dl_v), _p(self.dl_H), _p(self.u), _p(self.v), _p(self.H),
                _p(self.phi), _p(self.mask), _p(self.ar_u), _p(self.ar_v), _p(self.ar_H), _p(self.bed),
                _p(self.B), _p(self.beta), _p(self.gamma), *self._phys(dt), *self._tail(), _f(cfg.ssa_damping),
                _f(cfg.mc_damping), stream), "vanka_smooth_adjoint")
            self.l_u -= w * self.dl_u
            self.l_v -= w * self.dl_v
            self.l_H -= w * self.dl_H

    def gradients(self, stream=None):
        for which, g in ((0, self.g_beta), (1, self.g_bed)):
            g.fill_(0)
            _check(lib().grg_compute_gradient(
                which, *self._geom(), _p(g), _p(self.u), _p(self.v), _p(self.H), _p(self.l_u), _p(self.l_v),
                _p(self.l_H), _p(self.phi), _p(self.mask), _p(self.bed), _p(self.B), _p(self.beta), _p(self.gamma),
                *self._phys(0.0), *self._tail(), stream), "compute_gradient")


def _transfer(name, src, dst, ny, nx, total, stream=None):
    _check(lib().grg_transfer(TRANSFER[name], (total + 255) // 256, _p(src), _p(dst), ny, nx, stream), name)


def restrict_u(f, c):
    nyc, nxc = c.shape[0], c.shape[1] - 1
    _transfer("restrict_vfacet", f, c, nyc, nxc, nyc * (nxc + 1))


def restrict_v(f, c):
    nyc, nxc = c.shape[0] - 1, c.shape[1]
    _transfer("restrict_hfacet", f, c, nyc, nxc, (nyc + 1) * nxc)


def restrict_cell(f, c, method="avg"):
    nyc, nxc = c.shape
    _transfer(f"restrict_cell_{method}", f, c, nyc, nxc, nyc * nxc)


def prolong_u(c, f, method="bilinear"):
    ny, nx = c.shape[0] * 2, (c.shape[1] - 1) * 2
    _transfer(f"prolongate_vfacet_{method}", c, f, ny, nx, ny * (nx + 1))


def prolong_v(c, f, method="bilinear"):
    # glide/multigrid.py:212-235: the u-face kernels on the v arrays
    ny, nx = (c.shape[0] - 1) * 2, c.shape[1] * 2
    _transfer(f"prolongate_vfacet_{method}", c, f, ny, nx, (ny + 1) * nx)


def prolong_cell(c, f, method="injection"):
    ny, nx = c.shape[0] * 2, c.shape[1] * 2
    _transfer(f"prolongate_cell_{method}", c, f, ny, nx, ny * nx)


class RefGpuModel:
    """IceDynamics of the reference over its own GPU kernels."""

    def __init__(self, ny, nx, dx, n_levels, device="cuda"):
        if ny != nx:
            raise ValueError("the reference's v-face prolongation needs a square grid")
        self.levels = [RefLevel(ny, nx, dx, device)]
        for _ in range(1, n_levels):
            f = self.levels[-1]
            self.levels.append(RefLevel(f.ny // 2, f.nx // 2, f.dx * 2, device))
        self.fas = FASConfig()
        self.adj = FASConfig()
        self.dt = None
        self.history = []

    def set_field(self, name, value, start_level=0):
        """HierarchyFieldManager.set: set, then restrict to every coarser level
        (cell averages; max for the mask)."""
        lv = self.levels
        getattr(lv[start_level], name).copy_(torch.as_tensor(value, dtype=torch.float32))
        for l in range(start_level, len(lv) - 1):
            f, c = getattr(lv[l], name), getattr(lv[l + 1], name)
            if name == "u":
                restrict_u(f, c)
            elif name == "v":
                restrict_v(f, c)
            else:
                restrict_cell(f, c, "max" if name == "mask" else "avg")

    def restrict_state(self, f, c):
        restrict_u(f.u, c.u)
        restrict_v(f.v, c.v)
        restrict_cell(f.H, c.H)
        restrict_cell(f.H_prev, c.H_prev)
        restrict_cell(f.phi, c.phi)
        restrict_cell(f.mask, c.mask, "max")

    # -- forward: FASCDSolver.solve / vcycle --------------------------------
    def solve(self, dt, start_level=0):
        self.dt = float(torch.tensor(dt, dtype=torch.float32))
        top = self.levels[start_level]
        top.set_rhs(self.dt)
        ru, rv, rH = top.residual(self.dt, norms=True)
        r0 = torch.sqrt(ru ** 2 + rv ** 2 + rH ** 2)
        rel = torch.tensor(1.0, dtype=torch.float32)
        ab, it = r0, 0
        cfg = self.fas
        self.history = [float(r0)]
        while bool(rel > cfg.relative_tolerance) and bool(ab > cfg.absolute_tolerance) and it < cfg.maximum_vcycles:
            self.vcycle(start_level, finest=True)
            ru, rv, rH = top.residual(self.dt, freeze_phi=True, norms=True)
            ab = torch.sqrt(ru ** 2 + rv ** 2 + rH ** 2)
            rel = ab / r0
            self.history.append(float(ab))
            it += 1
        return it

    def _sweep(self, lev, n, coarse):
        cfg = self.fas
        lev.vanka_sweep(self.dt, n, freeze_calving=coarse and cfg.freeze_coarse_calving,
                        freeze_phi=coarse and cfg.freeze_coarse_phi)

    def vcycle(self, l, finest=False):
        coarse = not finest
        cfg = self.fas
        dt = self.dt
        lev = self.levels[l]
        if finest:
            lev.w_u[:, :] = lev.u
            lev.w_v[:, :] = lev.v
            lev.w_H[:, :] = lev.H
            lev.chi[:, :] = lev.phys["thklim"] - lev.H
        if l == len(self.levels) - 1:
            lev.gamma[:, :] = lev.w_H + lev.chi
            self._sweep(lev, cfg.coarsest_steps, coarse)
            lev.gamma.fill_(lev.phys["thklim"])
            return
        nxt = self.levels[l + 1]
        restrict_cell(lev.chi, nxt.chi, "max")
        prolong_cell(-nxt.chi, lev.phi_s, "injection")
        lev.phi_s[:, :] += lev.chi
        lev.gamma[:, :] = lev.w_H + lev.phi_s
        self._sweep(lev, cfg.pre_steps, coarse)
        lev.gamma.fill_(lev.phys["thklim"])
        lev.y_u[:, :] = lev.u - lev.w_u
        lev.y_v[:, :] = lev.v - lev.w_v
        lev.y_H[:, :] = lev.H - lev.w_H
        self.restrict_state(lev, nxt)
        nxt.w_u[:, :] = nxt.u
        nxt.w_v[:, :] = nxt.v
        nxt.w_H[:, :] = nxt.H
        lev.residual(dt, use_mask=False, freeze_calving=coarse and cfg.freeze_coarse_calving, freeze_phi=True)
        restrict_u(lev.r_u, nxt.r_u)
        restrict_v(lev.r_v, nxt.r_v)
        restrict_cell(lev.r_H, nxt.r_H)
        nxt.residual(dt, use_mask=False, operator_only=True, freeze_calving=cfg.freeze_coarse_calving,
                     freeze_phi=cfg.freeze_coarse_phi)
        nxt.f_u[:, :] = nxt.F_u - nxt.r_u
        nxt.f_v[:, :] = nxt.F_v - nxt.r_v
        nxt.f_H[:, :] = nxt.F_H - nxt.r_H
        self.vcycle(l + 1)
        nxt.z_u[:] = nxt.u - nxt.w_u
        nxt.z_v[:] = nxt.v - nxt.w_v
        nxt.z_H[:] = nxt.H - nxt.w_H
        prolong_u(nxt.z_u, lev.z_u, "bilinear")
        prolong_v(nxt.z_v, lev.z_v, "bilinear")
        prolong_cell(nxt.z_H, lev.z_H, "injection")
        lev.z_u[:, :] += lev.y_u
        lev.z_v[:, :] += lev.y_v
        lev.z_H[:, :] += lev.y_H
        lev.u[:, :] = lev.w_u + lev.z_u
        lev.v[:, :] = lev.w_v + lev.z_v
        lev.H[:, :] = lev.w_H + lev.z_H
        lev.gamma[:, :] = lev.w_H + lev.chi
        self._sweep(lev, cfg.post_steps, coarse)
        lev.gamma.fill_(lev.phys["thklim"])
        if finest:
            lev.vanka_sweep(dt, cfg.finest_steps)

    def forward(self, dt, update_geometry=True):
        """IceDynamics.forward (glide/model.py:65-72)."""
        it = self.solve(dt)
        if update_geometry:
            self.levels[0].H_prev[:, :] = self.levels[0].H
        return it

    # -- adjoint: FASAdjointSolver.solve / vcycle ---------------------------
    def adjoint_solve(self, dt, start_level=0):
        self.dt = float(torch.tensor(dt, dtype=torch.float32))
        top = self.levels[start_level]
        ru, rv, rH = top.adj_residual(self.dt, norms=True)
        r0 = torch.sqrt(ru ** 2 + rv ** 2 + rH ** 2)
        rel = torch.tensor(1.0, dtype=torch.float32)
        ab, it = r0, 0
        cfg = self.adj
        self.adj_history = [float(r0)]
        while bool(rel > cfg.relative_tolerance) and bool(ab > cfg.absolute_tolerance) and it < cfg.maximum_vcycles:
            self.adj_vcycle(start_level, finest=True)
            ru, rv, rH = top.adj_residual(self.dt, norms=True)
            ab = torch.sqrt(ru ** 2 + rv ** 2 + rH ** 2)
            rel = ab / r0
            self.adj_history.append(float(ab))
            it += 1
        return it

    def adj_vcycle(self, l, finest=False):
        cfg = self.adj
        dt = self.dt
        lev = self.levels[l]
        if l == len(self.levels) - 1:
            lev.adj_sweep(dt, cfg.coarsest_steps)
            return
        nxt = self.levels[l + 1]
        lev.adj_sweep(dt, cfg.pre_steps)
        self.restrict_state(lev, nxt)
        restrict_u(lev.l_u, nxt.l_u)
        restrict_v(lev.l_v, nxt.l_v)
        restrict_cell(lev.l_H, nxt.l_H)
        nxt.wl_u[:, :] = nxt.l_u
        nxt.wl_v[:, :] = nxt.l_v
        nxt.wl_H[:, :] = nxt.l_H
        lev.adj_residual(dt)
        restrict_u(lev.ar_u, nxt.ar_u)
        restrict_v(lev.ar_v, nxt.ar_v)
        restrict_cell(lev.ar_H, nxt.ar_H)
        nxt.adj_vjp(dt)
        nxt.af_u[:, :] = nxt.vjp_u - nxt.ar_u
        nxt.af_v[:, :] = nxt.vjp_v - nxt.ar_v
        nxt.af_H[:, :] = nxt.vjp_H - nxt.ar_H
        self.adj_vcycle(l + 1)
        nxt.zl_u[:, :] = nxt.l_u - nxt.wl_u
        nxt.zl_v[:, :] = nxt.l_v - nxt.wl_v
        nxt.zl_H[:, :] = nxt.l_H - nxt.wl_H
        prolong_u(nxt.zl_u, lev.zl_u, "bilinear")
        prolong_v(nxt.zl_v, lev.zl_v, "bilinear")
        prolong_cell(nxt.zl_H, lev.zl_H, "bilinear")
        lev.l_u[:, :] += lev.zl_u
        lev.l_v[:, :] += lev.zl_v
        lev.l_H[:, :] += lev.zl_H
        lev.adj_sweep(dt, cfg.post_steps)
        if finest:
            lev.adj_sweep(dt, cfg.finest_steps)

    def backward(self, dt, dJdu=None, dJdv=None, dJdH=None):
        """IceDynamics.backward (glide/model.py:74-94): adjoint solve, then
        the gradients with respect to beta and bed (H_prev and smb are the
        element-wise -lambda_H / dt and -lambda_H)."""
        top = self.levels[0]
        for arr, g in ((top.af_u, dJdu), (top.af_v, dJdv), (top.af_H, dJdH)):
            if g is None:
                arr.fill_(0.0)
            else:
                arr[:, :] = -g
        it = self.adjoint_solve(dt)
        top.gradients()
        dt32 = float(torch.tensor(dt, dtype=torch.float32))
        return it, {"beta": top.g_beta, "bed": top.g_bed, "H_prev": -top.l_H / dt32, "smb": -top.l_H}
