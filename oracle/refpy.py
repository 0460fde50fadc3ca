"""Run the reference's own Python package on host cores (test infrastructure).

The reference (JacobDowns/glide) imports CuPy at module top and compiles its
CUDA kernels with cupy.RawModule.  Neither CuPy nor a GPU is needed here:
`load_reference()` installs a NumPy-backed stand-in for the small part of the
CuPy API the package uses, plus an inert `xarray` stand-in (only used by its
I/O helpers), and routes every RawModule kernel launch to the reference's own
kernel sources compiled for the host (oracle/_ref/libglide_ref{32,64}.so, built
by oracle/build_oracle.py and executed by the fiber emulator in simt_host.cpp).

With fp64=True the stand-in maps `cupy.float32` to numpy.float64 and the kernels
come from the binary64 build, so the whole reference package -- its own
V-cycle sequencing, option objects, field managers and kernels -- runs in
binary64.  This is how the golden fixtures under tests/golden/ are produced and
how the oracle restatement is pinned.

Only this container has the reference checkout; nothing on a GPU box imports
this module.
"""
from __future__ import annotations

import ctypes
import importlib
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
DEFAULT_REFERENCE = os.environ.get("GLIDE_REFERENCE", "/root/reference")

# Kernel signatures: p = array pointer, b = bool, r = real scalar, i = int.
_P15 = "p" * 15
_PHYS = "r" * 11
_SIGS = {
    "compute_residual": ("2d", _P15 + "bb" + _PHYS + "iiii"),
    "compute_jvp": ("2d", "p" * 18 + "b" + _PHYS + "iiii"),
    "compute_vjp": ("2d", "p" * 18 + "bb" + _PHYS + "iiii"),
    "compute_grounded": ("2d", "ppp" + "rr" + "iiii"),
    "vanka_smooth": ("2d", "p" * 15 + _PHYS + "iiii" + "i" + "rrr"),
    "vanka_smooth_adjoint": ("2d", "p" * 15 + _PHYS + "iiii" + "rr"),
    "vanka_dump": ("2d", "p" * 13 + _PHYS + "iiii"),
    "compute_gradient_beta": ("2d", "p" * 13 + _PHYS + "iiii"),
    "compute_gradient_bed": ("2d", "p" * 13 + _PHYS + "iiii"),
}
_SIGS.update({
    "enthalpy_compute_residual": ("1d", "p" * 10 + "r" * 5 + "ii" + "iii"),
    "enthalpy_column_smooth": ("1d", "p" * 10 + "r" * 5 + "i" + "iii" + "ir"),
    "enthalpy_layer_smooth": ("1d", "p" * 10 + "r" * 5 + "i" + "iii"),
    "compute_omega": ("1d", "p" * 6 + "r" + "iii"),
})
for _name in ("restrict_vfacet", "restrict_hfacet", "restrict_cell_avg", "restrict_cell_max",
              "restrict_cell_min", "restrict_cell_var", "prolongate_vfacet_injection",
              "prolongate_vfacet_bilinear", "prolongate_hfacet_injection",
              "prolongate_hfacet_bilinear", "prolongate_cell_injection",
              "prolongate_cell_bilinear"):
    _SIGS[_name] = ("1d", "ppii")


class RefKernels:
    """ctypes view of one host build of the reference kernels."""

    def __init__(self, fp64: bool):
        self.fp64 = fp64
        self.real = np.float64 if fp64 else np.float32
        self.c_real = ctypes.c_double if fp64 else ctypes.c_float
        path = HERE / "_ref" / f"libglide_ref{64 if fp64 else 32}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run python oracle/build_oracle.py")
        self.lib = ctypes.CDLL(str(path))
        assert self.lib.gref_real_bytes() == (8 if fp64 else 4)

    def launch(self, name, grid, block, args):
        kind, sig = _SIGS[name]
        if len(sig) != len(args):
            raise TypeError(f"{name}: expected {len(sig)} args, got {len(args)}")
        grid = tuple(grid) if isinstance(grid, (tuple, list)) else (grid,)
        block = tuple(block) if isinstance(block, (tuple, list)) else (block,)
        if kind == "2d":
            head = [int(grid[0]), int(grid[1]) if len(grid) > 1 else 1,
                    int(block[0]), int(block[1]) if len(block) > 1 else 1]
        else:
            head = [int(grid[0]), int(block[0])]
        cargs = [ctypes.c_int(h) for h in head]
        keep = []
        for code, a in zip(sig, args):
            if code == "p":
                arr = a
                if not isinstance(arr, np.ndarray) or arr.dtype != self.real \
                        or not arr.flags.c_contiguous:
                    raise TypeError(f"{name}: array argument must be C-contiguous {self.real}")
                keep.append(arr)
                cargs.append(ctypes.c_void_p(arr.ctypes.data))
            elif code == "b":
                cargs.append(ctypes.c_bool(bool(a)))
            elif code == "r":
                cargs.append(self.c_real(float(a)))
            else:
                cargs.append(ctypes.c_int(int(a)))
        getattr(self.lib, "gref_" + name)(*cargs)


def _make_fake_cupy(kernels: RefKernels) -> types.ModuleType:
    cp = types.ModuleType("cupy")
    real = kernels.real

    def __getattr__(name):
        return getattr(np, name)

    cp.__getattr__ = __getattr__
    cp.float32 = real
    cp.float64 = np.float64
    cp.ndarray = np.ndarray
    cp.pi = np.pi
    cp.asnumpy = lambda a: np.asarray(a)
    cp.linalg = np.linalg
    cp.random = np.random

    class _Func:
        def __init__(self, name):
            self.name = name

        def __call__(self, grid, block, args, **kw):
            kernels.launch(self.name, grid, block, args)

    class RawModule:
        def __init__(self, code=None, options=(), **kw):
            self.options = options

        def get_function(self, name):
            if name not in _SIGS:
                raise NotImplementedError(f"kernel {name} is not wired into the host harness")
            return _Func(name)

    cp.RawModule = RawModule
    typing_mod = types.ModuleType("cupy.typing")
    typing_mod.NDArray = np.ndarray
    cp.typing = typing_mod
    cuda_mod = types.ModuleType("cupy.cuda")
    cp.cuda = cuda_mod
    return cp, typing_mod


def _make_fake_xarray() -> types.ModuleType:
    xr = types.ModuleType("xarray")

    class _Unavailable:
        def __init__(self, *a, **k):
            raise RuntimeError("xarray export is outside the solver path")

    xr.DataArray = _Unavailable
    xr.Dataset = _Unavailable
    return xr


def load_reference(fp64: bool = True, reference: str = DEFAULT_REFERENCE):
    """Import the reference `glide` package on host cores; returns the module.

    Importing twice with different precision re-imports the package.
    """
    kernels = RefKernels(fp64)
    cp, typing_mod = _make_fake_cupy(kernels)
    for k in [k for k in sys.modules if k == "glide" or k.startswith("glide.")]:
        del sys.modules[k]
    sys.modules["cupy"] = cp
    sys.modules["cupy.typing"] = typing_mod
    sys.modules["cupy.cuda"] = cp.cuda
    sys.modules.setdefault("xarray", _make_fake_xarray())
    if reference not in sys.path:
        sys.path.insert(0, reference)
    glide = importlib.import_module("glide")
    for sub in ("field", "grid", "operators", "multigrid", "model", "enthalpy"):
        importlib.import_module("glide." + sub)
    glide._kernels = kernels
    return glide
