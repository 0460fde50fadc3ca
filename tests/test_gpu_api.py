"""The reference-facing Python API on the GPU: IceDynamics, the field
managers and option objects, GlideStep (torch.autograd) and the IcePhysics
facade reproduce the reference's own C1 forward and adjoint (golden
fixtures made by running the reference's package) at 1e-10."""
from __future__ import annotations

import numpy as np
import pytest

from util import load_golden, rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FIELDS = ("bed", "B", "beta", "smb")


def _np(t):
    return t.detach().cpu().numpy()


def _model(g, quirks=True):
    from glide_b200.model import IceDynamics
    model = IceDynamics(n_levels=4, ny=64, nx=64, dx=1000.0, reference_quirks=quirks)
    mg = model.mg
    groups = {"bed": mg.geometry, "B": mg.rheology, "beta": mg.sliding, "smb": mg.forcing}
    for k in FIELDS:
        getattr(groups[k], k).set(torch.as_tensor(g[f"in_{k}"]))
    mg.state.H.set(torch.as_tensor(g["in_H"]))
    mg.state.H_prev.set(torch.as_tensor(g["in_H_prev"]))
    model.forward_solver.fas_options.set(maximum_vcycles=3, relative_tolerance=0.0, absolute_tolerance=0.0,
                                         report_norms=False)
    return model


def test_ice_dynamics_forward_matches_reference():
    g = load_golden("c1_forward_f64")
    model = _model(g)
    model.forward(0.0, 10.0, update_geometry=False)
    st = model.mg.levels[0].state
    for k in ("u", "v", "H", "mask", "phi"):
        assert rel_err(_np(getattr(st, k).data), g[f"out_{k}"]) <= 1e-10, k


def test_ice_dynamics_backward_matches_reference():
    g = load_golden("c1_adjoint_f64")
    model = _model(g)
    model.forward(0.0, 10.0, update_geometry=False)
    model.adjoint_solver.fas_options.set(maximum_vcycles=2, relative_tolerance=0.0, absolute_tolerance=0.0,
                                         report_norms=False)
    model.backward(0.0, 10.0, dJdu=torch.as_tensor(g["in_dJdu"]), dJdv=torch.as_tensor(g["in_dJdv"]))
    lv = model.mg.levels[0]
    for k in ("lambda_u", "lambda_v", "lambda_H"):
        assert rel_err(_np(getattr(lv.adjoint, k).data), g[f"out_{k}"]) <= 1e-10, k
    assert rel_err(_np(lv.sliding.beta.grad), g["out_grad_beta"]) <= 1e-10
    assert rel_err(_np(lv.geometry.bed.grad), g["out_grad_bed"]) <= 1e-10
    assert rel_err(_np(lv.state.H_prev.grad), g["out_grad_H_prev"]) <= 1e-10
    assert rel_err(_np(lv.forcing.smb.grad), g["out_grad_smb"]) <= 1e-10


def test_glide_step_autograd_matches_reference():
    """GlideStep.apply forward = IceDynamics.forward; its backward with output
    gradients (dJdu, dJdv, 0) returns the reference's parameter gradients."""
    from glide_b200.torch import GlideStep
    g = load_golden("c1_adjoint_f64")
    model = _model(g)
    model.adjoint_solver.fas_options.set(maximum_vcycles=2, relative_tolerance=0.0, absolute_tolerance=0.0,
                                         report_norms=False)
    dev = "cuda"
    leaf = {k: torch.as_tensor(g[f"in_{k}"], device=dev).requires_grad_(True)
            for k in ("H_prev", "bed", "beta", "smb")}
    u, v, H = GlideStep.apply(0.0, 10.0, model, 0, leaf["H_prev"], leaf["bed"], leaf["beta"], leaf["smb"])
    assert rel_err(_np(u), g["out_u"]) <= 1e-10
    assert rel_err(_np(H), g["out_H"]) <= 1e-10
    torch.autograd.backward([u, v], [torch.as_tensor(g["in_dJdu"], device=dev),
                                     torch.as_tensor(g["in_dJdv"], device=dev)])
    assert rel_err(_np(leaf["beta"].grad), g["out_grad_beta"]) <= 1e-10
    assert rel_err(_np(leaf["bed"].grad), g["out_grad_bed"]) <= 1e-10
    assert rel_err(_np(leaf["H_prev"].grad), g["out_grad_H_prev"]) <= 1e-10
    assert rel_err(_np(leaf["smb"].grad), g["out_grad_smb"]) <= 1e-10


def _converged_model(g):
    model = _model(g, quirks=False)
    model.forward_solver.fas_options.set(maximum_vcycles=100, relative_tolerance=1e-12, absolute_tolerance=0.0)
    model.adjoint_solver.fas_options.set(maximum_vcycles=100, relative_tolerance=1e-12, absolute_tolerance=0.0,
                                         report_norms=False)
    return model


def test_glide_step_two_steps_recompute_state():
    """Two chained steps through one model in native mode: each backward
    restores its own checkpointed forward state and starts its adjoint from
    lambda = 0, so the gradient of the summed loss equals the sum of the two
    steps' gradients computed on fresh models.  Solves are converged
    (truncated ones depend on their warm start)."""
    from glide_b200.torch import GlideStep
    g = load_golden("c1_adjoint_f64")
    dev = "cuda"
    H0 = torch.as_tensor(g["in_H_prev"], device=dev)
    bed = torch.as_tensor(g["in_bed"], device=dev)
    smb = torch.as_tensor(g["in_smb"], device=dev)
    model = _converged_model(g)
    beta = torch.as_tensor(g["in_beta"], device=dev).requires_grad_(True)
    u1, v1, H1 = GlideStep.apply(0.0, 10.0, model, 0, H0, bed, beta, smb)
    u2, v2, H2 = GlideStep.apply(10.0, 10.0, model, 0, H1.detach(), bed, beta, smb)
    ((u1 * 0.1).sum() + (u2 * 0.1).sum()).backward()
    per = []
    for Hin in (H0, H1.detach()):
        m = _converged_model(g)
        b = torch.as_tensor(g["in_beta"], device=dev).requires_grad_(True)
        uu, _, _ = GlideStep.apply(0.0, 10.0, m, 0, Hin, bed, b, smb)
        (uu * 0.1).sum().backward()
        per.append(b.grad.clone())
    assert rel_err(_np(beta.grad), _np(per[0] + per[1])) <= 1e-9


def test_ice_physics_facade():
    from glide_b200.physics import IcePhysics
    g = load_golden("c1_adjoint_f64")
    phys = IcePhysics(64, 64, 1000.0, 4)
    T = lambda k: torch.as_tensor(g[f"in_{k}"])
    phys.set_geometry(T("bed"), T("H"))
    phys.set_parameters(T("B"), T("beta"), T("smb"))
    u, v, H = phys.forward(10.0, n_vcycles=3)
    assert rel_err(_np(u), g["out_u"]) <= 1e-10
    grad = phys.adjoint(torch.as_tensor(g["in_dJdu"]), torch.as_tensor(g["in_dJdv"]), n_vcycles=2)
    assert rel_err(_np(grad), g["out_grad_beta"]) <= 1e-10


def test_unknown_option_raises():
    g = load_golden("c1_forward_f64")
    model = _model(g)
    with pytest.raises(AttributeError):
        model.forward_solver.fas_options.set(no_such_option=1)


def test_solver_vcycle_reproduces_reference_solves():
    """FASCDSolver.vcycle / FASAdjointSolver.vcycle called by hand, with the
    set-up their solve() does around them (right-hand side and phi; adjoint
    forcing), repeat the reference's 3-cycle forward and 2-cycle adjoint."""
    g = load_golden("c1_adjoint_f64")
    model = _model(g)
    lv = model.mg.levels[0]
    ops = lv.forward_operators
    ops.set_rhs(10.0)
    ops.compute_residual(10.0)
    fs = model.forward_solver
    with pytest.raises(AttributeError):
        fs.vcycle(0, finest=True)
    fs.dt = 10.0
    for _ in range(3):
        fs.vcycle(0, finest=True)
    for k in ("u", "v", "H"):
        assert rel_err(_np(getattr(lv.state, k).data), g[f"out_{k}"]) <= 1e-10, k
    aops = lv.adjoint_operators
    aops.f_u.copy_(-torch.as_tensor(g["in_dJdu"], device="cuda"))
    aops.f_v.copy_(-torch.as_tensor(g["in_dJdv"], device="cuda"))
    aops.f_H.zero_()
    adj = model.adjoint_solver
    adj.dt = 10.0
    for _ in range(2):
        adj.vcycle(0, finest=True)
    for k in ("lambda_u", "lambda_v", "lambda_H"):
        assert rel_err(_np(getattr(lv.adjoint, k).data), g[f"out_{k}"]) <= 1e-10, k


def test_adjoint_vanka_smooth_is_one_sweep():
    """AdjointOperators.vanka_smooth applies one adjoint smoother pass."""
    g = load_golden("c1_adjoint_f64")
    out = []
    for smooth in (True, False):
        model = _model(g)
        model.forward(0.0, 10.0, update_geometry=False)
        lv = model.mg.levels[0]
        lv.adjoint_operators.f_u.copy_(-torch.as_tensor(g["in_dJdu"], device="cuda"))
        lv.adjoint_operators.f_v.zero_()
        lv.adjoint_operators.f_H.zero_()
        if smooth:
            lv.adjoint_operators.vanka_smooth(10.0)
            lv.adjoint_operators.vanka_smooth(10.0)
        else:
            lv.adjoint_operators.vanka_sweep(10.0, 2)
        out.append(_np(lv.adjoint.lambda_u.data))
    assert np.abs(out[0]).max() > 0
    assert rel_err(out[0], out[1]) == 0.0


def test_not_converged_status_is_opt_in():
    """GLIDE_ERR_NOT_CONVERGED: off by default (the reference reports
    nothing); when on, a solve that stops at its cycle cap short of its
    tolerances raises NotConverged with its statistics, after writing every
    output; a solve that meets its tolerance does not raise."""
    from glide_b200._lib import GLIDE_ERR_NOT_CONVERGED, NotConverged
    g = load_golden("c1_forward_f64")
    model = _model(g)  # 3 cycles, zero tolerances: stops at the cap
    model.forward(0.0, 10.0, update_geometry=False)
    model = _model(g)
    model.mg.hierarchy.set_tuning(report_not_converged=True)
    with pytest.raises(NotConverged) as e:
        model.forward(0.0, 10.0, update_geometry=False)
    assert e.value.code == GLIDE_ERR_NOT_CONVERGED and e.value.stats["vcycles"] == 3
    st = model.mg.levels[0].state
    for k in ("u", "v", "H"):
        assert rel_err(_np(getattr(st, k).data), g[f"out_{k}"]) <= 1e-10, k
    ga = load_golden("c1_adjoint_f64")
    model.adjoint_solver.fas_options.set(maximum_vcycles=2, relative_tolerance=0.0, absolute_tolerance=0.0,
                                         report_norms=False)
    with pytest.raises(NotConverged):
        model.backward(0.0, 10.0, dJdu=torch.as_tensor(ga["in_dJdu"]), dJdv=torch.as_tensor(ga["in_dJdv"]))
    assert rel_err(_np(model.mg.levels[0].sliding.beta.grad), ga["out_grad_beta"]) <= 1e-10
    model = _model(g)
    model.mg.hierarchy.set_tuning(report_not_converged=True)
    model.forward_solver.fas_options.set(maximum_vcycles=100, relative_tolerance=1e-3)
    model.forward(0.0, 10.0, update_geometry=False)
