"""The one-field transfers of glide/multigrid.py:118-259 (restrict_vfacet,
restrict_hfacet, restrict_cell avg/max/min/var, prolongate_vfacet /
prolongate_hfacet / prolongate_cell with injection or bilinear weights).

CPU: the oracle's restatement against the fixture made by running the
reference's own Multigrid methods (tests/golden/transfers_f64.npz).
GPU: the Multigrid mirror's methods (glide_transfer through the C ABI)
against the same fixture, their argument errors, and the grid-level
helpers (create_coarse_grid, restrict_state ... restrict_residual).
"""
from __future__ import annotations

import numpy as np
import pytest

from util import load_golden, rel_err

TAGS = ("sq", "rect")
METHODS = ("injection", "bilinear")


@pytest.fixture(scope="module")
def g():
    return load_golden("transfers_f64")


@pytest.fixture(scope="module")
def _built():
    from oracle import build_oracle
    build_oracle.build_oracle()


def _oracle_outputs(g, tag):
    from oracle import glide_oracle as go
    fu, fv, fc = g[f"{tag}_fine_u"], g[f"{tag}_fine_v"], g[f"{tag}_fine_c"]
    cu, cv, cc = g[f"{tag}_coarse_u"], g[f"{tag}_coarse_v"], g[f"{tag}_coarse_c"]
    out = {}
    o = np.empty_like(cu); go._restrict_u(fu, o); out["restrict_vfacet"] = o
    o = np.empty_like(cv); go._restrict_v(fv, o); out["restrict_hfacet"] = o
    for m in ("avg", "max", "min", "var"):
        o = np.empty_like(cc); go._restrict_cell(fc, o, m); out[f"restrict_cell_{m}"] = o
    for m in METHODS:
        b = m == "bilinear"
        o = np.empty_like(fu); go._prolong_u(cu, o, b); out[f"prolongate_vfacet_{m}"] = o
        o = np.empty_like(fc); go._prolong_cell(cc, o, b); out[f"prolongate_cell_{m}"] = o
        o = np.empty_like(fv); go._prolong_v(cv, o, b); out[f"vface_prolongate_hfacet_{m}"] = o
        if fc.shape[0] == fc.shape[1]:
            o = np.empty_like(fv); go._prolong_v_as_reference(cv, o, b); out[f"prolongate_hfacet_{m}"] = o
    return out


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_transfers_match_reference(g, _built, tag):
    out = _oracle_outputs(g, tag)
    assert len(out) >= 12
    for k, v in out.items():
        assert rel_err(v, g[f"{tag}_{k}"]) <= 1e-15, k


# ----------------------------------------------------------------- GPU
def _mg(quirks=True, n=16):
    from glide_b200.multigrid import Multigrid
    return Multigrid(2, ny=n, nx=n, dx=1000.0, reference_quirks=quirks)


def _T(a, dtype=None):
    import torch
    return torch.as_tensor(a, device="cuda", dtype=dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", TAGS)
def test_gpu_transfers_match_reference(g, tag):
    mg, mg_native = _mg(True), _mg(False)
    fu, fv, fc = (_T(g[f"{tag}_fine_{k}"]) for k in "uvc")
    cu, cv, cc = (_T(g[f"{tag}_coarse_{k}"]) for k in "uvc")
    got = {"restrict_vfacet": mg.restrict_vfacet(fu), "restrict_hfacet": mg.restrict_hfacet(fv)}
    for m in ("avg", "max", "min", "var"):
        got[f"restrict_cell_{m}"] = mg.restrict_cell(fc, method=m)
    for m in METHODS:
        got[f"prolongate_vfacet_{m}"] = mg.prolongate_vfacet(cu, method=m)
        got[f"prolongate_cell_{m}"] = mg.prolongate_cell(cc, method=m)
        got[f"vface_prolongate_hfacet_{m}"] = mg_native.prolongate_hfacet(cv, method=m)
        if tag == "sq":
            got[f"prolongate_hfacet_{m}"] = mg.prolongate_hfacet(cv, method=m)
    for k, v in got.items():
        ref = g[f"{tag}_{k}"]
        assert tuple(v.shape) == ref.shape, k
        assert rel_err(v.cpu().numpy(), ref) <= 1e-15, k


@pytest.mark.gpu
def test_gpu_transfers_binary32_and_strided_outputs(g):
    """binary32 inputs give binary32 outputs within binary32 rounding of the
    binary64 reference; an output that is a strided view (a slice of a wider
    array) is written in place, leaving the rest of its storage untouched."""
    import torch
    mg = _mg()
    fc = _T(g["sq_fine_c"], torch.float32)
    out = mg.restrict_cell(fc, method="var")
    assert out.dtype == torch.float32
    assert rel_err(out.cpu().numpy(), g["sq_restrict_cell_var"]) <= 1e-6
    big = torch.full((8, 20), 7.0, device="cuda", dtype=torch.float64)
    view = big[:, 3:12]
    mg.restrict_vfacet(_T(g["sq_fine_u"]), view)
    assert rel_err(view.cpu().numpy(), g["sq_restrict_vfacet"]) <= 1e-15
    assert bool((big[:, :3] == 7.0).all()) and bool((big[:, 12:] == 7.0).all())


@pytest.mark.gpu
def test_gpu_transfer_argument_errors(g):
    from glide_b200._lib import GlideError
    mg = _mg()
    fc = _T(g["rect_fine_c"])
    with pytest.raises(TypeError):
        mg.restrict_cell(fc, method="median")
    with pytest.raises(TypeError):
        mg.prolongate_cell(_T(g["rect_coarse_c"]), method="cubic")
    with pytest.raises(ValueError):
        mg.restrict_cell(fc, _T(np.zeros((3, 3))))
    # the reference's v-face prolongation reuses its u-face kernel: square only
    with pytest.raises(GlideError):
        mg.prolongate_hfacet(_T(g["rect_coarse_v"]))
    # odd fine cell counts have no exact halving
    with pytest.raises(GlideError):
        mg.restrict_cell(_T(np.zeros((5, 6))))


def _fill_grid(grid, rng):
    import torch
    for grp, names in (("state", ("u", "v", "H", "H_prev", "phi", "mask")), ("geometry", ("bed",)),
                       ("rheology", ("B",)), ("sliding", ("beta",)), ("forcing", ("smb",))):
        for k in names:
            f = getattr(getattr(grid, grp), k)
            f.set(torch.as_tensor(rng.standard_normal(tuple(f.data.shape))))


@pytest.mark.gpu
def test_gpu_create_coarse_grid_restricts_every_group():
    """create_coarse_grid (glide/multigrid.py:62-79) on a stand-alone Grid:
    the child has half the cells, twice dx, the shifted origin, the
    restricted fields (oracle transfers) and the parent's constants."""
    from glide_b200.grid import Grid
    from oracle import build_oracle
    from oracle import glide_oracle as go
    build_oracle.build_oracle()
    rng = np.random.default_rng(5)
    mg = _mg()
    parent = Grid(12, 20, 500.0, x0=10.0, y0=90.0)
    _fill_grid(parent, rng)
    parent.geometry.thklim.set(2.5)
    parent.sliding.m.set(1.0 / 3.0)
    parent.calving.calving_rate.set(4.0)
    child = mg.create_coarse_grid(parent)
    assert (child.ny, child.nx, child.dx) == (6, 10, 1000.0)
    assert (child.x0, child.y0) == (10.0 + 250.0, 90.0 - 250.0)
    assert parent.child is child and child.parent is parent
    spawned = Grid(8, 12, 100.0).spawn_child()
    assert (spawned.ny, spawned.nx, spawned.dx) == (4, 6, 200.0) and spawned.parent.child is spawned
    assert child.geometry.thklim.value == 2.5 and child.sliding.m.value == 1.0 / 3.0
    assert child.calving.calving_rate.value == 4.0
    np_ = lambda f: np.ascontiguousarray(f.data.detach().cpu().numpy())
    o = np.empty((6, 11)); go._restrict_u(np_(parent.state.u), o)
    assert rel_err(np_(child.state.u), o) <= 1e-15
    o = np.empty((7, 10)); go._restrict_v(np_(parent.state.v), o)
    assert rel_err(np_(child.state.v), o) <= 1e-15
    for grp, k, how in (("state", "H", "avg"), ("state", "mask", "max"), ("geometry", "bed", "avg"),
                        ("rheology", "B", "avg"), ("sliding", "beta", "avg"), ("forcing", "smb", "avg")):
        o = np.empty((6, 10))
        go._restrict_cell(np_(getattr(getattr(parent, grp), k)), o, how)
        assert rel_err(np_(getattr(getattr(child, grp), k)), o) <= 1e-15, k


@pytest.mark.gpu
def test_gpu_create_grid_hierarchy_and_restrict_residual():
    import torch
    rng = np.random.default_rng(9)
    mg = _mg(n=32)
    _fill_grid(mg.levels[0], rng)
    levels = mg.create_grid_hierarchy(2)
    assert levels is mg.levels
    fine, coarse = mg.levels
    expect = mg.restrict_cell(fine.state.H.data)
    assert rel_err(coarse.state.H.data.cpu().numpy(), expect.cpu().numpy()) == 0.0
    with pytest.raises(ValueError):
        mg.create_grid_hierarchy(3)
    for k in ("r_u", "r_v", "r_H"):
        getattr(fine.forward_operators, k).copy_(torch.as_tensor(
            rng.standard_normal(tuple(getattr(fine.forward_operators, k).shape))))
    mg.restrict_residual(fine, coarse)
    fo, co = fine.forward_operators, coarse.forward_operators
    assert rel_err(co.r_u.cpu().numpy(), mg.restrict_vfacet(fo.r_u).cpu().numpy()) == 0.0
    assert rel_err(co.r_v.cpu().numpy(), mg.restrict_hfacet(fo.r_v).cpu().numpy()) == 0.0
    assert rel_err(co.r_H.cpu().numpy(), mg.restrict_cell(fo.r_H).cpu().numpy()) == 0.0
