"""Python handle over one device hierarchy of the C ABI.

`Hierarchy` owns a `glide_handle`: the multigrid levels' arrays live in one
device arena allocated by the library; `view(field, level)` returns a torch
tensor that aliases the arena (zero copy, row pitch preserved as a stride).
All calls run on torch's current CUDA stream.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import FIELD_ID, call


def _solve_status(code: int, st) -> None:
    """Raise for a failed forward / backward call; NotConverged carries the
    solve's statistics."""
    if code == _lib.GLIDE_ERR_NOT_CONVERGED:
        msg = _lib.load().glide_last_error()
        raise _lib.NotConverged(msg.decode() if msg else "", st.to_dict())
    _lib.check(code)


def _stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def transfer(op: str, src: torch.Tensor, dst: torch.Tensor, ny_fine: int, nx_fine: int):
    """One glide_transfer (restriction or prolongation of one field) between
    two 2-D CUDA tensors of one float dtype with unit column stride."""
    for t in (src, dst):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.ndim == 2):
            raise TypeError("transfers take 2-D CUDA tensors")
        if t.stride(1) != 1 and t.shape[1] > 1:
            raise ValueError("transfers need rows with unit stride")
    if src.dtype != dst.dtype or src.dtype not in (torch.float64, torch.float32):
        raise TypeError("source and destination must both be float64 or both float32")
    dtype = _lib.GLIDE_F64 if src.dtype == torch.float64 else _lib.GLIDE_F32
    call("glide_transfer", _lib.TRANSFER_OPS[op], dtype, int(ny_fine), int(nx_fine),
         ctypes.c_void_p(src.data_ptr()), max(src.stride(0), src.shape[1]), ctypes.c_void_p(dst.data_ptr()),
         max(dst.stride(0), dst.shape[1]), _stream_ptr())


class _DeviceBuffer:
    """__cuda_array_interface__ adaptor so torch can alias arena memory."""

    def __init__(self, ptr, rows, cols, pitch, dtype, owner):
        itemsize = 8 if dtype == torch.float64 else 4
        self.__cuda_array_interface__ = {
            "shape": (rows, cols),
            "strides": (pitch * itemsize, itemsize),
            "typestr": "<f8" if dtype == torch.float64 else "<f4",
            "data": (ptr, False),
            "version": 3,
        }
        self._owner = owner


class Hierarchy:
    def __init__(self, ny: int, nx: int, dx: float, n_levels: int, dtype=torch.float64,
                 reference_quirks: bool = True, use_graphs: bool = True, precision: str | None = None):
        """precision: "fp64" (default for float64), "fp32", or "mixed" (binary64
        fields and residuals, binary32 smoother and coarse levels)."""
        if not torch.cuda.is_available():
            raise _lib.GlideError(_lib.GLIDE_ERR_STATE, "glide_b200 needs a CUDA device (sm_100a)")
        if precision is None:
            precision = "fp64" if dtype == torch.float64 else "fp32"
        codes = {"fp64": _lib.GLIDE_F64, "fp32": _lib.GLIDE_F32, "mixed": _lib.GLIDE_MIXED}
        if precision not in codes:
            raise ValueError("precision must be 'fp64', 'fp32' or 'mixed'")
        dtype = torch.float32 if precision == "fp32" else torch.float64
        self.dtype = dtype
        self.precision = precision
        self.n_levels = n_levels
        lib = _lib.load()
        h = ctypes.c_void_p()
        torch.cuda.init()
        _lib.check(lib.glide_create(int(ny), int(nx), float(dx), int(n_levels), codes[precision],
                                    ctypes.byref(h)))
        self._h = h
        self._views = {}
        self.shapes = []
        for l in range(n_levels):
            a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
            call("glide_level_shape", h, l, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
            self.shapes.append((a.value, b.value, c.value))
        self.set_reference_quirks(reference_quirks)
        self.set_use_graphs(use_graphs)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize()
                _lib.load().glide_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    # -- field access --------------------------------------------------
    def view(self, field: str, level: int) -> torch.Tensor:
        key = (field, level)
        t = self._views.get(key)
        if t is None:
            p, r, c, pt = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            call("glide_field_ptr", self._h, FIELD_ID[field], int(level), ctypes.byref(p),
                 ctypes.byref(r), ctypes.byref(c), ctypes.byref(pt))
            buf = _DeviceBuffer(p.value, r.value, c.value, pt.value, self.dtype, self)
            t = torch.as_tensor(buf, device="cuda")
            self._views[key] = t
        return t

    def set(self, field: str, level: int, value, restrict_down: bool = False):
        """Copy `value` (tensor/array or scalar) into a level's field."""
        if isinstance(value, (int, float)) or (hasattr(value, "ndim") and getattr(value, "ndim") == 0
                                                and not isinstance(value, torch.Tensor)):
            call("glide_fill_field", self._h, FIELD_ID[field], int(level), float(value),
                 int(restrict_down), _stream_ptr())
            return
        t = torch.as_tensor(value)
        if t.ndim == 0:
            call("glide_fill_field", self._h, FIELD_ID[field], int(level), float(t.item()),
                 int(restrict_down), _stream_ptr())
            return
        dst = self.view(field, level)
        if tuple(t.shape) != tuple(dst.shape):
            raise ValueError(f"{field}: expected shape {tuple(dst.shape)}, got {tuple(t.shape)}")
        t = t.to(device="cuda", dtype=self.dtype).contiguous()
        call("glide_set_field", self._h, FIELD_ID[field], int(level), ctypes.c_void_p(t.data_ptr()),
             t.shape[1], 0, int(restrict_down), _stream_ptr())

    def get(self, field: str, level: int) -> torch.Tensor:
        return self.view(field, level).clone()

    def restrict(self, field: str, level: int):
        call("glide_restrict_field", self._h, FIELD_ID[field], int(level), _stream_ptr())

    # -- configuration -------------------------------------------------
    def get_phys(self, level: int) -> dict:
        p = _lib.Phys()
        call("glide_get_phys", self._h, int(level), ctypes.byref(p))
        return {k: getattr(p, k) for k, _ in _lib.Phys._fields_}

    def set_phys(self, level: int, **kw):
        levels = range(self.n_levels) if level < 0 else [level]
        for l in levels:
            cur = self.get_phys(l)
            cur.update({k: float(v) for k, v in kw.items()})
            call("glide_set_phys", self._h, l, ctypes.byref(_lib.Phys(**cur)))

    def get_fas(self, adjoint: bool) -> dict:
        c = _lib.FasConfig()
        call("glide_get_fas_config", self._h, int(adjoint), ctypes.byref(c))
        return {k: getattr(c, k) for k, _ in _lib.FasConfig._fields_}

    def set_fas(self, adjoint: bool, **kw):
        cur = self.get_fas(adjoint)
        cur.update(kw)
        cur = {k: (int(v) if t is ctypes.c_int else float(v)) for (k, t), v in
               zip(_lib.FasConfig._fields_, [cur[k] for k, _ in _lib.FasConfig._fields_])}
        call("glide_set_fas_config", self._h, int(adjoint), ctypes.byref(_lib.FasConfig(**cur)))

    def get_vanka(self, adjoint: bool, level: int) -> dict:
        c = _lib.VankaConfig()
        call("glide_get_vanka_config", self._h, int(adjoint), int(level), ctypes.byref(c))
        return {k: getattr(c, k) for k, _ in _lib.VankaConfig._fields_}

    def set_vanka(self, adjoint: bool, level: int, **kw):
        levels = range(self.n_levels) if level < 0 else [level]
        for l in levels:
            cur = self.get_vanka(adjoint, l)
            cur.update(kw)
            cur = {k: (int(cur[k]) if t is ctypes.c_int else float(cur[k])) for k, t in _lib.VankaConfig._fields_}
            call("glide_set_vanka_config", self._h, int(adjoint), l, ctypes.byref(_lib.VankaConfig(**cur)))

    def set_reference_quirks(self, on: bool):
        call("glide_set_reference_quirks", self._h, int(bool(on)))
        self.reference_quirks = bool(on)

    def set_use_graphs(self, on: bool):
        call("glide_set_use_graphs", self._h, int(bool(on)))

    def set_tuning(self, sweep_blocks_per_sm: int | None = None, mixed_inner_vcycles: int | None = None,
                   forward_method: str | None = None, newton_switch_exp10: int | None = None,
                   tangent_vcycles: int | None = None, tma_staging: bool | None = None,
                   report_not_converged: bool | None = None, tma_give_up: bool | None = None):
        """Solver knobs with no counterpart in the reference (see glide_set_tuning).
        forward_method: "fascd" (the reference's V-cycles only) or "newton"
        (FASCD until 10^-newton_switch_exp10, then Newton steps whose correction
        comes from the tangent linear multigrid).  report_not_converged: forward
        and backward raise NotConverged (with the solve's stats, after writing
        every output) when a solve stops at its cycle cap short of its
        tolerances; off by default, as the reference reports nothing.
        tma_give_up: every stencil block's first wait for its staged tiles
        gives up at once, so the call fails with GLIDE_ERR_TIMEOUT (a test of
        that path; the blocks still let their copies land before returning)."""
        if sweep_blocks_per_sm is not None:
            call("glide_set_tuning", self._h, _lib.TUNE_SWEEP_BLOCKS_PER_SM, int(sweep_blocks_per_sm))
        if mixed_inner_vcycles is not None:
            call("glide_set_tuning", self._h, _lib.TUNE_MIXED_INNER_VCYCLES, int(mixed_inner_vcycles))
        if forward_method is not None:
            call("glide_set_tuning", self._h, _lib.TUNE_FORWARD_METHOD, {"fascd": 0, "newton": 1}[forward_method])
        if newton_switch_exp10 is not None:
            call("glide_set_tuning", self._h, _lib.TUNE_NEWTON_SWITCH_EXP10, int(newton_switch_exp10))
        if tangent_vcycles is not None:
            call("glide_set_tuning", self._h, _lib.TUNE_TANGENT_VCYCLES, int(tangent_vcycles))
        if tma_staging is not None:
            call("glide_set_tuning", self._h, _lib.TUNE_TMA_STAGING, int(bool(tma_staging)))
        if report_not_converged is not None:
            call("glide_set_tuning", self._h, _lib.TUNE_REPORT_NOT_CONVERGED, int(bool(report_not_converged)))
        if tma_give_up is not None:
            call("glide_set_tuning", self._h, _lib.TUNE_TMA_GIVE_UP, int(bool(tma_give_up)))

    def launch_count(self) -> int:
        c = ctypes.c_longlong()
        call("glide_launch_count", self._h, ctypes.byref(c))
        return c.value

    def alg_bytes(self) -> float:
        """Algorithmic bytes of every kernel launched so far (glide_alg_bytes)."""
        c = ctypes.c_double()
        call("glide_alg_bytes", self._h, ctypes.byref(c))
        return c.value

    # -- operators -----------------------------------------------------
    def set_rhs(self, level: int, dt: float):
        call("glide_set_rhs", self._h, int(level), float(dt), _stream_ptr())

    def compute_phi(self, level: int, relaxation: float = 0.0):
        call("glide_compute_phi", self._h, int(level), float(relaxation), _stream_ptr())

    def residual(self, level: int, dt: float, flags: int, norms: bool = False):
        out = (ctypes.c_double * 3)() if norms else None
        call("glide_residual", self._h, int(level), float(dt), int(flags), out, _stream_ptr())
        return tuple(out) if norms else None

    def vanka_sweep(self, level: int, dt: float, n: int, flags: int = 0, newton_iters=None):
        p = ctypes.c_void_p(newton_iters.data_ptr()) if newton_iters is not None else None
        call("glide_vanka_sweep", self._h, int(level), float(dt), int(n), int(flags), p, _stream_ptr())

    def vanka_dump(self, level: int, dt: float):
        """Local 5x5 Vanka systems (J (ny*nx, 25), r (ny*nx, 5)) of every cell."""
        ny, nx, _ = self.shapes[level]
        J = torch.empty((ny * nx, 25), dtype=self.dtype, device="cuda")
        r = torch.empty((ny * nx, 5), dtype=self.dtype, device="cuda")
        call("glide_vanka_dump", self._h, int(level), float(dt), ctypes.c_void_p(J.data_ptr()),
             ctypes.c_void_p(r.data_ptr()), _stream_ptr())
        return J, r

    def forward(self, dt: float, start_level: int = 0) -> dict:
        st = _lib.Stats()
        _solve_status(_lib.load().glide_forward(self._h, float(dt), int(start_level), ctypes.byref(st),
                                                _stream_ptr()), st)
        return st.to_dict()

    def adjoint_residual(self, level: int, dt: float, norms: bool = False):
        out = (ctypes.c_double * 3)() if norms else None
        call("glide_adjoint_residual", self._h, int(level), float(dt), out, _stream_ptr())
        return tuple(out) if norms else None

    def vjp(self, level: int, dt: float):
        call("glide_vjp", self._h, int(level), float(dt), _stream_ptr())

    def jvp(self, level: int, dt: float, reference_rows: bool = True, flags: int = _lib.USE_MASK):
        """flags: USE_MASK (the default) and FREEZE_CALVING, as glide_jvp."""
        call("glide_jvp", self._h, int(level), float(dt), int(bool(reference_rows)), int(flags), _stream_ptr())

    def block_factor(self, level: int, dt: float, adjoint: bool = False):
        """One launch of the linear smoother's block factorisation alone
        (glide_block_smoother_part; instrumentation)."""
        call("glide_block_smoother_part", self._h, int(level), float(dt), int(bool(adjoint)), 0, _stream_ptr())

    def block_sweep(self, level: int, dt: float, adjoint: bool = False):
        """One launch of the linear smoother's block sweep alone."""
        call("glide_block_smoother_part", self._h, int(level), float(dt), int(bool(adjoint)), 1, _stream_ptr())

    def adjoint_sweep(self, level: int, dt: float, n: int):
        call("glide_adjoint_sweep", self._h, int(level), float(dt), int(n), _stream_ptr())

    def gradients(self, level: int, dt: float, mask: int = _lib.GRAD_ALL):
        call("glide_gradients", self._h, int(level), float(dt), int(mask), _stream_ptr())

    def vcycle(self, adjoint: bool, level: int, finest: bool, dt: float):
        """One V-cycle from `level` (no residual around it; see glide_vcycle)."""
        call("glide_vcycle", self._h, int(bool(adjoint)), int(level), int(bool(finest)), float(dt), _stream_ptr())

    def backward(self, dt: float, start_level: int = 0, mask: int = _lib.GRAD_ALL) -> dict:
        st = _lib.Stats()
        _solve_status(_lib.load().glide_backward(self._h, float(dt), int(start_level), int(mask),
                                                 ctypes.byref(st), _stream_ptr()), st)
        return st.to_dict()
