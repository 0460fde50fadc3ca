"""Chains of GlideSteps with the forward states checkpointed and recomputed.

1. Gradients of a loss over a chain of steps are bit-identical whether every
   step's solved state is kept (the reference's behaviour) or only every k-th
   one is and the backward pass re-solves the others, in reference mode (the
   adjoint warm-started from the previous lambda) and native mode.
2. The C3 configuration as specified: a 20-step chain on the 512^2 dome,
   loss sum over steps of 0.5 sum((u - u_obs)^2 + (v - v_obs)^2) with the
   observations from a chain with beta perturbed by a seeded 30 % log-normal
   factor, every 5th state kept; grad-beta against central finite differences
   along 8 seeded directions at steps 1e-2 ... 1e-6 (the best step within
   5 %, the tolerance of the reference's tests/grad_test.py: its transpose
   applies the forward viscosity derivative), and the mixed-precision
   gradient against the binary64 one (1e-6).
"""
from __future__ import annotations

import numpy as np
import pytest

from cases import dome
from util import rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _model(f, n, dx, levels, precision="fp64", quirks=True, rtol=1e-10, fast=False):
    from glide_b200.ensemble import CANDIDATES, apply_schedule
    from glide_b200.model import IceDynamics
    m = IceDynamics(n_levels=levels, ny=n, nx=n, dx=dx, reference_quirks=quirks, precision=precision)
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


def _chain(m, f, beta, bed, n_steps, dt, obs=None):
    """n_steps GlideSteps from rest; returns the outputs and the loss
    sum_k 0.5 |u_k - uo_k|^2 + |v_k - vo_k|^2 (0 without observations)."""
    from glide_b200.torch import GlideStep
    for k in ("u", "v", "mask"):
        getattr(m.mg.state, k).set(0.0)
    H = torch.as_tensor(f["H"], device="cuda")
    smb = torch.as_tensor(f["smb"], device="cuda")
    outs, loss = [], 0.0
    for k in range(n_steps):
        u, v, H = GlideStep.apply(k * dt, dt, m, 0, H, bed, beta, smb)
        outs.append((u, v))
        if obs is not None:
            uo, vo = obs[k]
            loss = loss + 0.5 * (((u - uo) ** 2).sum() + ((v - vo) ** 2).sum())
    return outs, loss


@pytest.mark.parametrize("quirks", [True, False])
def test_recomputed_states_give_bit_identical_gradients(quirks):
    from glide_b200.torch import checkpointing
    n, dx, levels, dt, steps = 128, 6000.0, 4, 10.0, 7
    f = dome(n, dx, 300e3, seed=4)
    rng = np.random.default_rng(9)
    obs = [(torch.as_tensor(rng.normal(0, 20, (n, n + 1)), device="cuda"),
            torch.as_tensor(rng.normal(0, 20, (n + 1, n)), device="cuda")) for _ in range(steps)]
    grads, policies = {}, {}
    for every in (1, 3, 7):
        m = _model(f, n, dx, levels, quirks=quirks)
        policies[every] = checkpointing(m, every=every)
        beta = torch.as_tensor(f["beta"], device="cuda").clone().requires_grad_(True)
        bed = torch.as_tensor(f["bed"], device="cuda").clone().requires_grad_(True)
        _, loss = _chain(m, f, beta, bed, steps, dt, obs)
        loss.backward()
        grads[every] = (beta.grad.clone(), bed.grad.clone())
        del m
    for every in (3, 7):
        assert torch.equal(grads[every][0], grads[1][0]), every
        assert torch.equal(grads[every][1], grads[1][1]), every
    p3, p7 = policies[3], policies[7]
    assert (p3.kept_steps, p3.dropped_steps) == (3, 4)  # steps 0, 3, 6 kept
    assert p3.recomputed_steps == 4
    assert (p7.kept_steps, p7.dropped_steps) == (1, 6)
    assert p7.recomputed_steps == 6  # one segment, re-solved once


def test_c3_twenty_step_gradient_matches_finite_differences():
    from glide_b200.torch import checkpointing
    n, dx, levels, dt, steps = 512, 1500.0, 5, 10.0, 20
    f = dome(n, dx, 600e3, seed=0)
    rng = np.random.default_rng(42)
    beta0 = torch.as_tensor(f["beta"], device="cuda")
    bed = torch.as_tensor(f["bed"], device="cuda")
    m = _model(f, n, dx, levels, quirks=False, rtol=1e-12, fast=True)
    pert = torch.as_tensor(np.exp(0.3 * rng.standard_normal(f["beta"].shape)), device="cuda")
    with torch.no_grad():
        outs, _ = _chain(m, f, beta0 * pert, bed, steps, dt)
    obs = [(u.clone(), v.clone()) for u, v in outs]

    def loss_at(beta):
        with torch.no_grad():
            return float(_chain(m, f, beta, bed, steps, dt, obs)[1])

    policy = checkpointing(m, every=5)
    beta = beta0.clone().requires_grad_(True)
    _, loss = _chain(m, f, beta, bed, steps, dt, obs)
    loss.backward()
    g = beta.grad.clone()
    assert policy.kept_steps == 4 and policy.recomputed_steps == 16
    worst = 0.0
    for d in range(8):
        dirn = torch.as_tensor(rng.standard_normal(f["beta"].shape), device="cuda") * beta0
        adj = float((g * dirn).sum())
        best = np.inf
        for h in (1e-2, 1e-3, 1e-4, 1e-5, 1e-6):
            fd = (loss_at(beta0 + h * dirn) - loss_at(beta0 - h * dirn)) / (2 * h)
            best = min(best, abs(adj - fd) / max(abs(fd), 1e-300))
        worst = max(worst, best)
    print(f"C3 20-step grad-beta vs central FD: worst best-step relative error {worst:.3e}")
    assert worst <= 5e-2, worst

    # the same chain with the mixed-precision form
    mm = _model(f, n, dx, levels, precision="mixed", quirks=False, rtol=1e-12, fast=True)
    checkpointing(mm, every=5)
    beta_m = beta0.clone().requires_grad_(True)
    _, loss_m = _chain(mm, f, beta_m, bed, steps, dt, obs)
    loss_m.backward()
    err = rel_err(beta_m.grad.cpu().numpy(), g.cpu().numpy())
    print(f"C3 20-step grad-beta, mixed vs binary64: {err:.3e}")
    assert err <= 1e-6, err
