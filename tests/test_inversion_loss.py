"""The inversion objective of glide_b200.inversion (the reference's
examples/greenland/greenland_inverse.py:131-155) on CPU tensors, against a
direct NumPy evaluation of the same formula; and the ensemble's convergence
test of a forward solve."""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_inversion_loss_matches_formula():
    from glide_b200.inversion import InversionLoss
    rng = np.random.default_rng(0)
    ny, nx, dx = 12, 10, 750.0
    u = rng.standard_normal((ny, nx + 1))
    v = rng.standard_normal((ny + 1, nx))
    uo = rng.standard_normal((ny, nx))
    vo = rng.standard_normal((ny, nx))
    uo[0, :3] = 0.0  # below the mask threshold: not in the misfit
    lb = rng.standard_normal((ny, nx))
    loss = InversionLoss(l2=1e-3, tv=2e-4, eps=1e-6, mask_threshold=0.01)
    J, jd, j1, j2 = loss(*(torch.as_tensor(x) for x in (u, v, uo, vo, lb)), dx)
    uc, vc = 0.5 * (u[:, 1:] + u[:, :-1]), 0.5 * (v[1:] + v[:-1])
    mu, mv = np.abs(uo) > 0.01, np.abs(vo) > 0.01
    ref_d = (np.abs(uc - uo) * mu).mean() + (np.abs(vc - vo) * mv).mean()
    gy, gx = np.diff(lb, axis=0) / dx, np.diff(lb, axis=1) / dx
    ref_2 = 1e-3 * ((gy ** 2).sum() + (gx ** 2).sum()) * dx ** 2
    ref_1 = 2e-4 * np.sqrt(gy[:, :-1] ** 2 + gx[:-1] ** 2 + 1e-12).sum() * dx ** 2
    assert abs(float(jd) - ref_d) <= 1e-12 * abs(ref_d)
    assert abs(float(j2) - ref_2) <= 1e-12 * abs(ref_2)
    assert abs(float(j1) - ref_1) <= 1e-12 * abs(ref_1)
    assert abs(float(J) - (ref_d + ref_1 + ref_2)) <= 1e-12 * abs(float(J))


def test_inversion_loss_gradient_reaches_log_beta():
    from glide_b200.inversion import InversionLoss
    lb = torch.zeros(6, 5, dtype=torch.float64)
    lb[2, 3] = 1.0
    lb.requires_grad_(True)
    J, *_ = InversionLoss(l2=1.0, tv=0.0)(torch.zeros(6, 6, dtype=torch.float64),
                                          torch.zeros(7, 5, dtype=torch.float64),
                                          torch.zeros(6, 5, dtype=torch.float64),
                                          torch.zeros(6, 5, dtype=torch.float64), lb, 1.0)
    J.backward()
    # d/dx of sum of squared first differences: 2 * (number of neighbours) at the bump
    assert float(lb.grad[2, 3]) == pytest.approx(8.0)


def test_ensemble_convergence_rule():
    from types import SimpleNamespace
    from glide_b200.ensemble import _converged
    m = SimpleNamespace(forward_solver=SimpleNamespace(
        _fas_config=SimpleNamespace(relative_tolerance=1e-8, absolute_tolerance=0.0)))
    assert _converged(m, {"initial_norm": 1.0, "final_norm": 1e-8})
    assert not _converged(m, {"initial_norm": 1.0, "final_norm": 2e-8})
    m.forward_solver._fas_config.absolute_tolerance = 1e-3
    assert _converged(m, {"initial_norm": 1.0, "final_norm": 5e-4})
