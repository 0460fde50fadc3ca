"""End-to-end checks on the configurations of the workload specification.

C2: the 512^2 dome (dx 1500 m, 5 levels, dt 10 a), 20 coupled steps, each
solved to a relative residual of 1e-10: the mixed-precision fast form stays
within 1e-6 (u, v) and 1e-8 (H) of the binary64 reference form.

C3: on the same dome, the adjoint gradient of
L = 0.5 sum((u - u_obs)^2 + (v - v_obs)^2) with respect to beta, u_obs from a
solve with beta perturbed by a seeded 30 % log-normal factor, against central
finite differences of L along 8 seeded directions at steps 1e-2 ... 1e-6: the
best step agrees within 5 % (the tolerance of the reference's tests/grad_test.py;
the reference's transpose applies the forward viscosity derivative, so the
adjoint gradient is close to, not equal to, the true one).
"""
from __future__ import annotations

import numpy as np
import pytest

from cases import dome
from util import rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N, DX, LEVELS, DT = 512, 1500.0, 5, 10.0


def _model(f, precision="fp64", quirks=True, fast=False, rtol=1e-10):
    from glide_b200.ensemble import CANDIDATES, apply_schedule
    from glide_b200.model import IceDynamics
    m = IceDynamics(n_levels=LEVELS, ny=N, nx=N, dx=DX, reference_quirks=quirks, precision=precision)
    mg = m.mg
    for k, grp in (("bed", mg.geometry), ("B", mg.rheology), ("beta", mg.sliding), ("smb", mg.forcing)):
        getattr(grp, k).set(torch.as_tensor(f[k]))
    mg.state.H.set(torch.as_tensor(f["H"]))
    mg.state.H_prev.set(torch.as_tensor(f["H_prev"]))
    if fast:
        apply_schedule(m, CANDIDATES["fast"])
    m.forward_solver.fas_options.set(maximum_vcycles=200, relative_tolerance=rtol, absolute_tolerance=0.0,
                                     report_norms=False)
    m.adjoint_solver.fas_options.set(maximum_vcycles=200, relative_tolerance=rtol, absolute_tolerance=0.0,
                                     report_norms=False)
    return m


def _state(m):
    st = m.mg.levels[0].state
    return {k: getattr(st, k).data.detach().cpu().numpy().copy() for k in ("u", "v", "H")}


def test_c2_twenty_steps_mixed_matches_binary64():
    f = dome(N, DX, 600e3, seed=0)
    ref = _model(f)
    fast = _model(f, precision="mixed", quirks=False, fast=True)
    for step in range(20):
        for m in (ref, fast):
            st = m.forward(step * DT, DT)
            assert st["final_norm"] <= 1e-10 * st["initial_norm"] or st["final_norm"] < 1e-9, (step, st)
    a, b = _state(fast), _state(ref)
    assert rel_err(a["u"], b["u"]) <= 1e-6
    assert rel_err(a["v"], b["v"]) <= 1e-6
    assert rel_err(a["H"], b["H"]) <= 1e-8


def _solve(m, f, beta):
    """One step from rest with the given beta."""
    mg = m.mg
    mg.sliding.beta.set(torch.as_tensor(beta))
    mg.state.H.set(torch.as_tensor(f["H"]))
    mg.state.H_prev.set(torch.as_tensor(f["H_prev"]))
    for k in ("u", "v"):
        getattr(mg.state, k).set(0.0)
    m.forward(0.0, DT, update_geometry=False)


def _loss_and_grad(m, f, beta, uo, vo, grad=True):
    mg = m.mg
    _solve(m, f, beta)
    s = mg.levels[0].state
    u, v = s.u.data.detach().clone(), s.v.data.detach().clone()
    du, dv = u - torch.as_tensor(uo, device="cuda"), v - torch.as_tensor(vo, device="cuda")
    L = 0.5 * float((du * du).sum() + (dv * dv).sum())
    if not grad:
        return L, None
    m.backward(0.0, DT, dJdu=du, dJdv=dv)
    return L, mg.levels[0].sliding.beta.grad.detach().cpu().numpy().copy()


def test_c3_adjoint_gradient_matches_finite_differences():
    f = dome(N, DX, 600e3, seed=0)
    rng = np.random.default_rng(42)
    beta0 = np.asarray(f["beta"])
    m = _model(f, quirks=False, rtol=1e-12)
    _solve(m, f, beta0 * np.exp(0.3 * rng.standard_normal(beta0.shape)))
    obs = _state(m)
    uo, vo = obs["u"], obs["v"]
    L0, g = _loss_and_grad(m, f, beta0, uo, vo)
    worst = 0.0
    for d in range(8):
        dirn = rng.standard_normal(beta0.shape) * beta0
        adj = float((g * dirn).sum())
        best = np.inf
        for h in (1e-2, 1e-3, 1e-4, 1e-5, 1e-6):
            Lp, _ = _loss_and_grad(m, f, beta0 + h * dirn, uo, vo, grad=False)
            Lm, _ = _loss_and_grad(m, f, beta0 - h * dirn, uo, vo, grad=False)
            fd = (Lp - Lm) / (2 * h)
            best = min(best, abs(adj - fd) / max(abs(fd), 1e-300))
        worst = max(worst, best)
    assert worst <= 5e-2, worst


def test_c3_dome_512_matches_reference():
    """The reference algorithm at the C3 size (512^2, 5 levels, its defaults
    and quirks): 3 forward V-cycles, then the adjoint of dJ/du = 0.05 u,
    dJ/dv = 0.05 v with 2 V-cycles and the gradients, against the
    reference's own run (fixture tests/golden/c3_dome512_f64.npz: values on a
    stride-7 lattice and each field's max-norm) at 1e-10."""
    from util import load_golden
    g = load_golden("c3_dome512_f64")
    f = dome(N, DX, 600e3, seed=0)
    for k in ("bed", "B", "beta", "smb", "H"):  # the regenerated inputs are the fixture's
        np.testing.assert_allclose([np.sum(f[k]), np.sum(np.abs(f[k]))], g[f"in_sum_{k}"], rtol=1e-13)
    m = _model(f)
    m.forward_solver.fas_options.set(maximum_vcycles=3, relative_tolerance=0.0, absolute_tolerance=0.0)
    m.forward(0.0, DT, update_geometry=False)
    st = m.mg.levels[0].state
    u, v = st.u.data.clone(), st.v.data.clone()
    m.adjoint_solver.fas_options.set(maximum_vcycles=2, relative_tolerance=0.0, absolute_tolerance=0.0)
    m.backward(0.0, DT, dJdu=0.05 * u, dJdv=0.05 * v)
    lv = m.mg.levels[0]
    got = {"u": st.u.data, "v": st.v.data, "H": st.H.data, "lambda_u": lv.adjoint.lambda_u.data,
           "lambda_v": lv.adjoint.lambda_v.data, "lambda_H": lv.adjoint.lambda_H.data,
           "grad_beta": lv.sliding.beta.grad, "grad_bed": lv.geometry.bed.grad}
    for k, t in got.items():
        a = t.detach().cpu().numpy()[::7, ::7]
        err = float(np.abs(a - g[f"out_{k}"]).max()) / float(g[f"max_{k}"])
        assert err <= 1e-10, (k, err)
