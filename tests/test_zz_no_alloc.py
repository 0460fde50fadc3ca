"""glide_residual_norms_noalloc against glide_residual, through the C ABI.

The no-allocation entry point launches the same residual kernel as the handle
API on caller-owned arrays, so residuals and norms must agree bit for bit.
Two calls in a row, with the outputs poisoned in between, show that the
static scratch needs no clearing and that every output is rewritten.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from util import load_golden

torch = pytest.importorskip("torch")

DT = 5.0


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _noalloc(lib, ny, nx, dx, phys, ins, flags, outs, norms, stream):
    return lib.glide_residual_norms_noalloc(
        ny, nx, dx, DT, ctypes.byref(phys),
        _ptr(ins["u"]), nx + 1, _ptr(ins["v"]), nx, _ptr(ins["H"]), _ptr(ins["phi"]), _ptr(ins["mask"]),
        _ptr(ins["f_u"]), _ptr(ins["f_v"]), _ptr(ins["f_H"]), _ptr(ins["bed"]), _ptr(ins["B"]),
        _ptr(ins["beta"]), _ptr(ins["gamma"]), nx, flags,
        _ptr(outs["r_u"]), _ptr(outs["r_v"]), _ptr(outs["r_H"]), _ptr(norms), stream)


@pytest.mark.gpu
def test_noalloc_residual_matches_handle_residual_twice():
    from glide_b200 import _lib
    from glide_b200.hierarchy import Hierarchy

    g = load_golden("random_residual_f64")
    ny, nx = g["in_H"].shape
    dx = 1500.0
    h = Hierarchy(ny, nx, dx, 1, precision="fp64", reference_quirks=True)
    for k in ("u", "v", "H", "H_prev", "mask", "bed", "B", "beta", "smb", "f_u", "f_v"):
        h.set(k, 0, torch.as_tensor(g[f"in_{k}"]))
    h.set_rhs(0, DT)
    flags = _lib.USE_MASK
    lib = _lib.load()
    phys = _lib.Phys(**h.get_phys(0))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    # inputs as plain contiguous tensors owned by the caller (phi is in/out)
    ins = {k: h.get(k, 0).contiguous() for k in
           ("u", "v", "H", "phi", "mask", "f_u", "f_v", "f_H", "bed", "B", "beta", "gamma")}
    outs = {k: torch.empty_like(h.view(k, 0)).contiguous() for k in ("r_u", "r_v", "r_H")}
    norms = torch.empty(4, dtype=torch.float64, device="cuda")

    for call_no in range(2):
        ref_norms = h.residual(0, DT, flags, norms=True)
        ref = {k: h.get(k, 0) for k in ("r_u", "r_v", "r_H", "phi")}
        for t in (*outs.values(), norms):
            t.fill_(float("nan"))
        ins["phi"].fill_(-1.0)  # finite garbage: recomputed from H and bed
        rc = _noalloc(lib, ny, nx, dx, phys, ins, flags, outs, norms, stream)
        assert rc == _lib.GLIDE_OK, (rc, lib.glide_noalloc_last_error())
        torch.cuda.synchronize()
        for k in ("r_u", "r_v", "r_H"):
            assert torch.equal(outs[k], ref[k]), (call_no, k)
        assert torch.equal(ins["phi"], ref["phi"]), call_no
        got = norms.cpu().numpy()
        np.testing.assert_array_equal(got[:3], np.array(ref_norms), err_msg=f"call {call_no}")
        assert got[3] == pytest.approx(float(np.sqrt(np.sum(np.square(ref_norms)))), rel=1e-14)


def test_noalloc_rejects_grids_beyond_its_scratch():
    """Sizes are checked before any pointer is touched or CUDA is called."""
    from glide_b200 import _lib
    lib = _lib.load()
    phys = _lib.Phys()
    fake = ctypes.c_void_p(256)  # never dereferenced: the size check comes first

    def call(ny, nx, ld_u, ld_v, ld_c):
        return lib.glide_residual_norms_noalloc(
            ny, nx, 1000.0, DT, ctypes.byref(phys), fake, ld_u, fake, ld_v, fake, fake, fake, fake, fake,
            fake, fake, fake, fake, fake, ld_c, 0, fake, fake, fake, fake, None)

    # too many tiles
    assert call(4097, 4097, 4098, 4097, 4097) == _lib.GLIDE_ERR_SHAPE
    assert b"4096 x 4096" in lib.glide_noalloc_last_error()
    # few tiles, but more rows than one launch's grid can hold
    assert call(70000, 16, 17, 16, 16) == _lib.GLIDE_ERR_SHAPE
    assert b"65535 rows" in lib.glide_noalloc_last_error()
    # nx near INT_MAX: nx + 1 must not wrap around and pass the pitch check
    big = 2**31 - 1
    assert call(16, big, -(2**31), big, big) == _lib.GLIDE_ERR_SHAPE
    assert b"ld_u >= nx + 1" in lib.glide_noalloc_last_error()
    # ... nor may the tile count wrap when every pitch is large enough
    assert call(16, big - 1, big, big - 1, big - 1) == _lib.GLIDE_ERR_SHAPE
    assert b"tiles" in lib.glide_noalloc_last_error()
