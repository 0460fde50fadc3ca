"""Pin the CPU oracle (oracle/glide_oracle.*) against the golden fixtures
produced by the reference itself (tests/golden/make_golden.py), and -- where
the reference checkout is present -- against the reference run live."""
from __future__ import annotations

import os

import numpy as np
import pytest

from util import load_golden, oracle_c1, oracle_single_level, rel_err

DT_RANDOM = 5.0


@pytest.fixture(scope="module", autouse=True)
def _built():
    from oracle import build_oracle
    build_oracle.build_oracle()


def test_c1_forward_matches_reference_f64():
    g = load_golden("c1_forward_f64")
    o = oracle_c1(g)
    o.fas.maximum_vcycles = 3
    o.fas.relative_tolerance = 0.0
    o.fas.absolute_tolerance = 0.0
    assert o.solve(10.0) == 3
    lev = o.levels[0]
    for k in ("u", "v", "H", "mask", "phi"):
        assert rel_err(getattr(lev, k), g[f"out_{k}"]) <= 1e-13, k


def test_c1_forward_matches_reference_f32():
    g = load_golden("c1_forward_f32")
    o = oracle_c1(g, dtype=np.float32)
    o.fas.maximum_vcycles = 3
    o.fas.relative_tolerance = 0.0
    o.fas.absolute_tolerance = 0.0
    o.solve(10.0)
    lev = o.levels[0]
    for k in ("u", "v", "H"):
        assert rel_err(getattr(lev, k), g[f"out_{k}"]) <= 1e-5, k


def test_c1_adjoint_matches_reference_f64():
    g = load_golden("c1_adjoint_f64")
    o = oracle_c1(g)
    o.fas.maximum_vcycles = 3
    o.fas.relative_tolerance = 0.0
    o.fas.absolute_tolerance = 0.0
    o.solve(10.0)
    o.adj.maximum_vcycles = 2
    o.adj.relative_tolerance = 0.0
    o.adj.absolute_tolerance = 0.0
    grads = o.backward(10.0, dJdu=g["in_dJdu"], dJdv=g["in_dJdv"])
    lev = o.levels[0]
    assert rel_err(lev.l_u, g["out_lambda_u"]) <= 1e-12
    assert rel_err(lev.l_v, g["out_lambda_v"]) <= 1e-12
    assert rel_err(lev.l_H, g["out_lambda_H"]) <= 1e-12
    for k in ("beta", "bed", "H_prev", "smb"):
        assert rel_err(grads[k], g[f"out_grad_{k}"]) <= 1e-12, k


def test_c1_adjoint_solution_depends_on_the_smoother_in_reference_mode():
    """A property of the reference's adjoint, shown on the oracle pinned to
    it.  The reference prolongates v-face corrections with its u-face kernel
    run on the v arrays, which writes into the pinned v faces (rows 0 and
    ny).  The adjoint residual leaves pinned rows out and the adjoint sweep
    zeroes their right-hand side, so nothing brings those values back: two
    solves of the C1 adjoint that converge the residual to 1e-12 under
    different smoother weights end at different lambda (about 2 % next to the
    domain edges, 0.1 % inside; the bed gradient moves by about 2 %).  With
    the corrected transfers (native mode) the pinned faces stay zero and the
    two solves agree to rounding.  This is why the binary32 adjoint smoothers
    keep binary32 block factors: in reference mode, rounding the factors
    moves the converged adjoint the same way."""
    from cases import slab_c1
    from oracle.glide_oracle import OracleHierarchy
    f = slab_c1()

    def run(omega, quirks):
        o = OracleHierarchy(64, 64, 1000.0, 4, reference_quirks=quirks)
        for k in ("bed", "B", "beta", "smb", "H", "H_prev"):
            o.set_field(k, f[k])
        o.fas.maximum_vcycles, o.fas.relative_tolerance, o.fas.absolute_tolerance = 30, 1e-11, 0.0
        o.solve(10.0)
        top = o.levels[0]
        o.adj.maximum_vcycles, o.adj.relative_tolerance, o.adj.absolute_tolerance = 200, 1e-12, 0.0
        for lev in o.levels:
            lev.adj_vanka.omega = omega
        g = o.backward(10.0, dJdu=0.1 * top.u, dJdv=0.1 * top.v)
        assert o.adj_history[-1] <= 1e-12 * o.adj_history[0]
        return top.l_v.copy(), g["bed"]

    lv_a, bed_a = run(0.5, True)
    lv_b, bed_b = run(0.8, True)
    assert rel_err(lv_b, lv_a) >= 1e-3
    assert rel_err(bed_b, bed_a) >= 1e-3
    assert np.abs(lv_a[[0, -1]]).max() >= 1e-3 * np.abs(lv_a).max()  # the pinned v faces moved
    lv_a, bed_a = run(0.5, False)
    lv_b, bed_b = run(0.8, False)
    assert rel_err(lv_b, lv_a) <= 1e-10
    assert rel_err(bed_b, bed_a) <= 1e-10
    assert np.abs(lv_a[[0, -1]]).max() == 0.0


@pytest.mark.parametrize("tag,calving", [("", 0.0), ("_calving", 2.0)])
def test_random_residual_matches_reference(tag, calving):
    g = load_golden("random_residual_f64")
    o = oracle_single_level(g, 1500.0, calving=calving)
    lev = o.levels[0]
    lev.f_H[...] = lev.H_prev / DT_RANDOM + lev.smb
    lev.residual(DT_RANDOM, use_mask=True)
    for k in ("r_u", "r_v", "r_H", "phi"):
        assert rel_err(getattr(lev, k), g[f"out_{k}{tag}"]) <= 1e-13, k
    lev.residual(DT_RANDOM, use_mask=False, operator_only=True, freeze_phi=True)
    for k in ("F_u", "F_v", "F_H"):
        assert rel_err(getattr(lev, k), g[f"out_{k}{tag}"]) <= 1e-13, k


def test_random_vanka_matches_reference():
    g = load_golden("random_vanka_f64")
    o = oracle_single_level(g, 1500.0)
    lev = o.levels[0]
    lev.f_H[...] = lev.H_prev / DT_RANDOM + lev.smb
    lev.vanka_sweep(DT_RANDOM, 3)
    for k in ("u", "v", "H", "mask", "phi"):
        assert rel_err(getattr(lev, k), g[f"out_{k}"]) <= 1e-12, k


def test_random_adjoint_matches_reference():
    g = load_golden("random_adjoint_f64")
    o = oracle_single_level(g, 1500.0)
    lev = o.levels[0]
    lev.compute_phi()
    lev.l_u[...], lev.l_v[...], lev.l_H[...] = g["in_lambda_u"], g["in_lambda_v"], g["in_lambda_H"]
    lev.af_u[...], lev.af_v[...], lev.af_H[...] = g["in_adj_f_u"], g["in_adj_f_v"], g["in_adj_f_H"]
    lev.adj_vjp(DT_RANDOM)
    for k in ("vjp_u", "vjp_v", "vjp_H"):
        assert rel_err(getattr(lev, k), g[f"out_{k}"]) <= 1e-12, k
    lev.adj_residual(DT_RANDOM)
    assert rel_err(lev.ar_u, g["out_adj_r_u"]) <= 1e-12
    assert rel_err(lev.ar_v, g["out_adj_r_v"]) <= 1e-12
    assert rel_err(lev.ar_H, g["out_adj_r_H"]) <= 1e-12
    lev.adj_sweep(DT_RANDOM, 2)
    assert rel_err(lev.l_u, g["out_sweep_lambda_u"]) <= 1e-12
    assert rel_err(lev.l_v, g["out_sweep_lambda_v"]) <= 1e-12
    assert rel_err(lev.l_H, g["out_sweep_lambda_H"]) <= 1e-12
    lev.gradients()
    assert rel_err(lev.g_beta, g["out_grad_beta"]) <= 1e-12
    assert rel_err(lev.g_bed, g["out_grad_bed"]) <= 1e-12


REF = os.environ.get("GLIDE_REFERENCE", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "glide", "cuda")),
                    reason="reference checkout not present")
def test_oracle_matches_live_reference_on_new_seed():
    """Fresh random state (seed not used by the fixtures), reference run live."""
    import contextlib
    import io

    from cases import random_state
    from oracle import build_oracle
    from oracle.refpy import load_reference
    build_oracle.build_reference(REF)
    load_reference(fp64=True, reference=REF)
    from glide.grid import Grid
    st = random_state(24, 30, seed=123)
    with contextlib.redirect_stdout(io.StringIO()):
        gr = Grid(24, 30, 900.0)
    for k in ("u", "v", "H", "H_prev", "mask"):
        getattr(gr.state, k).set(st[k])
    gr.geometry.bed.set(st["bed"]); gr.rheology.B.set(st["B"])
    gr.sliding.beta.set(st["beta"]); gr.forcing.smb.set(st["smb"])
    gr.forward_operators.f_u[:, :] = st["f_u"]
    gr.forward_operators.f_v[:, :] = st["f_v"]
    gr.forward_operators.set_rhs(2.0)
    gr.forward_operators.vanka_sweep(2.0, 2)
    inp = {f"in_{k}": v for k, v in st.items()}
    o = oracle_single_level(inp, 900.0)
    lev = o.levels[0]
    lev.f_H[...] = lev.H_prev / 2.0 + lev.smb
    lev.vanka_sweep(2.0, 2)
    for k in ("u", "v", "H", "mask"):
        assert rel_err(getattr(lev, k), np.array(getattr(gr.state, k).data)) <= 1e-12, k


def test_vanka_dump_matches_reference():
    """ForwardOperators.vanka_dump on the random state (with calving)."""
    from oracle.glide_oracle import OracleLevel
    g = load_golden("random_vanka_dump_f64")
    ny, nx = g["in_H"].shape
    lev = OracleLevel(ny, nx, 1500.0, np.float64)
    for k in ("u", "v", "H", "bed", "B", "beta", "phi", "gamma", "f_u", "f_v"):
        getattr(lev, k)[...] = g[f"in_{k}"]
    lev.phys["calving_rate"] = 1.0
    lev.f_H[...] = g["in_H_prev"] / 5.0 + g["in_smb"]
    J, r = lev.vanka_dump(5.0)
    assert rel_err(J, g["out_J"]) <= 1e-12
    assert rel_err(r, g["out_r"]) <= 1e-12


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "glide", "cuda")),
                    reason="reference checkout not present")
def test_oracle_operators_match_live_reference_on_new_shape():
    """A non-square 28 x 44 state on a seed no fixture uses, the reference
    run live: the masked residual and the forcing-free operator with
    calving (1e-13), then the transpose product, adjoint residual, two
    adjoint sweeps and the beta / bed gradients (1e-12)."""
    import contextlib
    import io

    from cases import random_state
    from oracle import build_oracle
    from oracle.refpy import load_reference
    build_oracle.build_reference(REF)
    load_reference(fp64=True, reference=REF)
    from glide.grid import Grid
    st = random_state(28, 44, seed=321)
    ny, nx = st["H"].shape
    dt = 3.0

    def grid(calving):
        with contextlib.redirect_stdout(io.StringIO()):
            g = Grid(ny, nx, 1500.0)
        for k in ("u", "v", "H", "H_prev", "mask"):
            getattr(g.state, k).set(st[k])
        g.geometry.bed.set(st["bed"]); g.rheology.B.set(st["B"])
        g.sliding.beta.set(st["beta"]); g.forcing.smb.set(st["smb"])
        g.calving.calving_rate.set(calving)
        g.forward_operators.f_u[:, :] = st["f_u"]
        g.forward_operators.f_v[:, :] = st["f_v"]
        return g

    inp = {f"in_{k}": v for k, v in st.items()}
    g = grid(1.0)
    ops = g.forward_operators
    ops.set_rhs(dt)
    ops.compute_residual(dt, use_mask=True)
    lev = oracle_single_level(inp, 1500.0, calving=1.0).levels[0]
    lev.f_H[...] = lev.H_prev / dt + lev.smb
    lev.residual(dt, use_mask=True)
    for k in ("r_u", "r_v", "r_H"):
        assert rel_err(getattr(lev, k), np.array(getattr(ops, k))) <= 1e-13, k
    ops.compute_residual(dt, use_mask=False, operator_only=True, freeze_phi=True)
    lev.residual(dt, use_mask=False, operator_only=True, freeze_phi=True)
    for k in ("F_u", "F_v", "F_H"):
        assert rel_err(getattr(lev, k), np.array(getattr(ops, k))) <= 1e-13, k

    rng = np.random.default_rng(99)
    lam = dict(lambda_u=rng.normal(0, 1, (ny, nx + 1)), lambda_v=rng.normal(0, 1, (ny + 1, nx)),
               lambda_H=rng.normal(0, 1, (ny, nx)))
    af = dict(adj_f_u=rng.normal(0, 1, (ny, nx + 1)), adj_f_v=rng.normal(0, 1, (ny + 1, nx)),
              adj_f_H=rng.normal(0, 1, (ny, nx)))
    g = grid(0.0)
    g.forward_operators.compute_phi()
    for k, v in lam.items():
        getattr(g.adjoint, k).set(v)
    aops = g.adjoint_operators
    aops.f_u[:, :], aops.f_v[:, :], aops.f_H[:, :] = af["adj_f_u"], af["adj_f_v"], af["adj_f_H"]
    lev = oracle_single_level(inp, 1500.0).levels[0]
    lev.compute_phi()
    lev.l_u[...], lev.l_v[...], lev.l_H[...] = lam["lambda_u"], lam["lambda_v"], lam["lambda_H"]
    lev.af_u[...], lev.af_v[...], lev.af_H[...] = af["adj_f_u"], af["adj_f_v"], af["adj_f_H"]
    aops.compute_vjp(dt)
    lev.adj_vjp(dt)
    for k in ("vjp_u", "vjp_v", "vjp_H"):
        assert rel_err(getattr(lev, k), np.array(getattr(aops, k))) <= 1e-12, k
    aops.compute_residual(dt)
    lev.adj_residual(dt)
    for k, r in (("ar_u", "r_u"), ("ar_v", "r_v"), ("ar_H", "r_H")):
        assert rel_err(getattr(lev, k), np.array(getattr(aops, r))) <= 1e-12, k
    aops.vanka_sweep(dt, 2)
    lev.adj_sweep(dt, 2)
    for k, r in (("l_u", "lambda_u"), ("l_v", "lambda_v"), ("l_H", "lambda_H")):
        assert rel_err(getattr(lev, k), np.array(getattr(g.adjoint, r).data)) <= 1e-12, k
    aops.compute_gradient_beta()
    aops.compute_gradient_bed()
    lev.gradients()
    assert rel_err(lev.g_beta, np.array(g.sliding.beta.grad)) <= 1e-12
    assert rel_err(lev.g_bed, np.array(g.geometry.bed.grad)) <= 1e-12
