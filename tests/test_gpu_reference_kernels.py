"""The reference's own kernels, built unmodified for sm_100a and driven by the
restated host sequence of oracle/ref_gpu.py (the GPU baseline the bench's
reference arm times), reproduce the reference's C1 results:

- forward, 3 V-cycles, against the binary32 fixture made by the host build
  of the same sources: 2e-4 relative (the GPU build uses fast-math
  intrinsics, as the reference compiles its kernels; the host build rounds
  correctly);
- adjoint, 2 V-cycles after that forward, against the binary64 fixture:
  lambda and grad-beta within 1e-2 relative (binary32 against binary64).
"""
from __future__ import annotations

import pytest

from util import load_golden, rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _model(g):
    from oracle import ref_gpu
    if not ref_gpu.LIB_PATH.exists():
        pytest.skip("oracle/_ref/libglide_ref_gpu.so not built (no reference checkout at build time)")
    m = ref_gpu.RefGpuModel(64, 64, 1000.0, 4)
    for k in ("bed", "B", "beta", "smb", "H", "H_prev"):
        m.set_field(k, torch.as_tensor(g[f"in_{k}"], device="cuda"))
    m.fas.maximum_vcycles, m.fas.relative_tolerance, m.fas.absolute_tolerance = 3, 0.0, 0.0
    return m


def test_reference_kernels_reproduce_c1_forward():
    g = load_golden("c1_forward_f32")
    m = _model(g)
    assert m.forward(10.0, update_geometry=False) == 3
    lev = m.levels[0]
    errs = {k: rel_err(getattr(lev, k).cpu().numpy(), g[f"out_{k}"]) for k in ("u", "v", "H")}
    print("reference kernels on the GPU vs the binary32 fixture:", errs)
    for k, e in errs.items():
        assert e <= 2e-4, (k, e)


def test_reference_kernels_c1_adjoint():
    g = load_golden("c1_adjoint_f64")
    m = _model(g)
    m.forward(10.0, update_geometry=False)
    m.adj.maximum_vcycles, m.adj.relative_tolerance, m.adj.absolute_tolerance = 2, 0.0, 0.0
    dev = lambda k: torch.as_tensor(g[k], dtype=torch.float32, device="cuda")
    it, grads = m.backward(10.0, dJdu=dev("in_dJdu"), dJdv=dev("in_dJdv"))
    assert it == 2
    lev = m.levels[0]
    errs = {k: rel_err(getattr(lev, a).cpu().numpy(), g[f"out_{k}"])
            for k, a in (("lambda_u", "l_u"), ("lambda_v", "l_v"), ("lambda_H", "l_H"))}
    errs["grad_beta"] = rel_err(grads["beta"].cpu().numpy(), g["out_grad_beta"])
    print("reference kernels on the GPU, adjoint vs the binary64 fixture:", errs)
    for k, e in errs.items():
        assert e <= 1e-2, (k, e)
