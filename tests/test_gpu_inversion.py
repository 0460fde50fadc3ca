"""The multi-level beta inversion driver (the reference's inverse example,
examples/greenland/greenland_inverse.py:71-175, as glide_b200.inversion):
observations from a known spatially varying beta on a 64 x 64 dome, the
inversion started from the uniform background beta at the coarsest of three
levels, must cut the finest level's velocity misfit well below that of the
uniform beta."""
from __future__ import annotations

import numpy as np
import pytest

from cases import dome

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N, DX, LEVELS, DT = 64, 2000.0, 3, 1.0


def _model(f):
    from glide_b200.model import IceDynamics
    m = IceDynamics(n_levels=LEVELS, ny=N, nx=N, dx=DX, reference_quirks=False)
    mg = m.mg
    for k, grp in (("bed", mg.geometry), ("B", mg.rheology), ("beta", mg.sliding), ("smb", mg.forcing)):
        getattr(grp, k).set(torch.as_tensor(f[k]))
    mg.state.H.set(torch.as_tensor(f["H"]))
    mg.state.H_prev.set(torch.as_tensor(f["H"]))
    for s in (m.forward_solver, m.adjoint_solver):
        s.fas_options.set(maximum_vcycles=30, relative_tolerance=1e-6, absolute_tolerance=0.0, report_norms=False)
    return m


def test_observation_hierarchy_is_cell_restriction():
    from glide_b200.inversion import observation_hierarchy
    f = dome(N, DX, 50e3, seed=1)
    m = _model(f)
    u = torch.rand(N, N, dtype=torch.float64, device="cuda")
    v = torch.rand(N, N, dtype=torch.float64, device="cuda")
    obs = observation_hierarchy(m.mg, u, v)
    assert [tuple(x.shape) for x, _ in obs] == [(64, 64), (32, 32), (16, 16)]
    ref = u.reshape(32, 2, 32, 2).mean(dim=(1, 3))
    assert float((obs[1][0] - ref).abs().max()) <= 1e-15


def test_inversion_reduces_velocity_misfit():
    from glide_b200.inversion import InversionLoss, invert_beta
    from glide_b200.torch import GlideStep
    f = dome(N, DX, 50e3, seed=1)
    x = (np.arange(N) + 0.5) / N
    pattern = np.sin(2 * np.pi * x)[:, None] * np.sin(2 * np.pi * x)[None, :]
    beta0 = np.asarray(f["beta"])
    beta_true = beta0 * np.exp(0.7 * pattern)
    m = _model(f)
    mg = m.mg
    dev = "cuda"
    H = torch.as_tensor(f["H"], device=dev)
    bed = torch.as_tensor(f["bed"], device=dev)
    smb = torch.as_tensor(f["smb"], device=dev)
    with torch.no_grad():
        u, v, _ = GlideStep.apply(0.0, DT, m, 0, H, bed, torch.as_tensor(beta_true, device=dev), smb)
        u_obs = (0.5 * (u[:, 1:] + u[:, :-1])).clone()
        v_obs = (0.5 * (v[1:] + v[:-1])).clone()
        loss = InversionLoss(l2=1e-9, tv=0.0)
        lb0 = torch.log(torch.as_tensor(beta0, device=dev))
        u0, v0, _ = GlideStep.apply(0.0, DT, m, 0, H, bed, torch.exp(lb0), smb)
        j0 = float(loss(u0, v0, u_obs, v_obs, lb0, DX)[1])
    assert j0 > 0
    mg.sliding.beta.set(torch.as_tensor(beta0))
    res = invert_beta(m, u_obs, v_obs, DT, coarsest_level=LEVELS - 1, epochs_per_level=20, loss=loss,
                      optimizer=lambda p: torch.optim.RMSprop(p, lr=0.05))
    assert [h[0] for h in res.history] == [2] * 20 + [1] * 20 + [0] * 20
    final = res.history[-1][3]
    assert np.isfinite(final) and final <= 0.5 * j0, (final, j0)
    assert tuple(res.log_beta.shape) == (N, N)
