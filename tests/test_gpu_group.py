"""Grouped solves (glide_b200.group): a group of uneven hierarchies runs each
kind of launch of a V-cycle once for all members, and every member computes
what its own solve computes: the same cycles, the same launches and
arguments.  The grouped kernels are separate compilations of the same tile
bodies, so the results agree to rounding (measured ~1e-12 relative after a
solve; asserted at the 1e-10 binary64 parity bar, in binary32 at ten times
the solve tolerance of 1e-4) and the cycle counts are identical.

- forward solves to a relative tolerance -- FASCD and guarded Newton with
  its undo and fallback decisions taken on the device -- members stopping at
  their own cycle counts, with different schedules in one group, over two
  time steps (plans replayed across steps);
- adjoint solves and gradients;
- binary64 and binary32;
and the merged cycle carries the members' launches in fewer grouped ones.
"""
from __future__ import annotations

import numpy as np
import pytest

from util import rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SIZES = [64, 96, 128, 64, 96]
LEVELS = [3, 3, 4, 3, 3]
SCHEDULES = ["fascd", "fast", "classic", "newton/classic", "fast"]
DT = 10.0


def _members(precision):
    from cases import dome
    from glide_b200.ensemble import CANDIDATES, apply_schedule
    from glide_b200.model import IceDynamics
    out = []
    for k, (n, L) in enumerate(zip(SIZES, LEVELS)):
        dx = 4000.0
        f = dome(n, dx, R=0.4 * n * dx, seed=30 + k)
        m = IceDynamics(n_levels=L, ny=n, nx=n, dx=dx, reference_quirks=False, precision=precision)
        mg = m.mg
        for key, grp in (("bed", mg.geometry), ("B", mg.rheology), ("beta", mg.sliding), ("smb", mg.forcing)):
            getattr(grp, key).set(torch.as_tensor(f[key]))
        mg.state.H.set(torch.as_tensor(f["H"]))
        mg.state.H_prev.set(torch.as_tensor(f["H_prev"]))
        # uneven schedules in one group: short FASCD, the classic 10/20/50/200,
        # guarded Newton with the tangent multigrid, and Newton falling back to
        # the classic schedule
        apply_schedule(m, CANDIDATES[SCHEDULES[k]])
        rtol = 1e-8 if precision == "fp64" else 1e-4
        m.forward_solver.fas_options.set(maximum_vcycles=60, relative_tolerance=rtol, absolute_tolerance=0.0,
                                         report_norms=False)
        m.adjoint_solver.fas_options.set(maximum_vcycles=40, relative_tolerance=rtol, absolute_tolerance=0.0,
                                         report_norms=False)
        out.append(m)
    return out


def _dJ(m):
    st = m.mg.levels[0].state
    return 0.05 * st.u.data, 0.05 * st.v.data, None


FIELDS = ("u", "v", "H", "mask", "phi", "lambda_u", "lambda_v", "lambda_H", "grad_beta", "grad_bed",
          "grad_H_prev", "grad_smb")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_group_matches_solo_solves(precision):
    from glide_b200.group import HierarchyGroup
    solo, grouped = _members(precision), _members(precision)
    solo_stats, group_stats = [], []
    for step in range(2):
        solo_stats.append([m.forward(step * DT, DT)["vcycles"] for m in solo])
    masks = []
    for m in solo:
        du, dv, dH = _dJ(m)
        solo_stats.append(m.backward(2 * DT, DT, dJdu=du, dJdv=dv)["vcycles"])
    g = HierarchyGroup([m.mg.hierarchy for m in grouped])
    for step in range(2):
        st = g.forward(DT)
        group_stats.append([s["vcycles"] for s in st])
        for m in grouped:
            lev = m.mg.levels[0]
            lev.state.H_prev.data.copy_(lev.state.H.data)
    for m in grouped:
        du, dv, dH = _dJ(m)
        masks.append(m.prepare_backward(dJdu=du, dJdv=dv))
    assert len(set(masks)) == 1
    bst = g.backward(DT, mask=masks[0])
    group_stats.extend(s["vcycles"] for s in bst)
    torch.cuda.synchronize()
    assert solo_stats == group_stats
    # the two forward steps stop after different cycle counts per member
    assert len(set(solo_stats[0])) > 1
    tol = 1e-10 if precision == "fp64" else 1e-3
    for a, b in zip(solo, grouped):
        for k in FIELDS:
            x = a.mg.hierarchy.get(k, 0).double().cpu().numpy()
            y = b.mg.hierarchy.get(k, 0).double().cpu().numpy()
            assert rel_err(y, x) <= tol, (k, rel_err(y, x))
    c = g.counters()
    grouped_launches, member_launches = c["forward_cycle"]
    assert grouped_launches < member_launches / 3, c
    g.close()


def test_group_refuses_mixed_members():
    from glide_b200 import _lib
    from glide_b200.group import HierarchyGroup
    from glide_b200.model import IceDynamics
    a = IceDynamics(n_levels=2, ny=32, nx=32, dx=4000.0, reference_quirks=False, precision="mixed")
    with pytest.raises(_lib.GlideError):
        HierarchyGroup([a.mg.hierarchy])
    b = IceDynamics(n_levels=2, ny=32, nx=32, dx=4000.0, reference_quirks=False)
    c = IceDynamics(n_levels=2, ny=32, nx=32, dx=4000.0, reference_quirks=False, precision="fp32")
    with pytest.raises(_lib.GlideError):
        HierarchyGroup([b.mg.hierarchy, c.mg.hierarchy])  # two precisions
    with pytest.raises(_lib.GlideError):
        HierarchyGroup([b.mg.hierarchy, b.mg.hierarchy])  # a handle twice


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_group_stops_on_staging_maps_that_fail_their_check(precision):
    """Staging maps in device memory that do not carry their tag are never
    handed to the TMA unit: the first stencil launch of each member records
    that in the member's error word, the member stops, and the call fails
    with GLIDE_ERR_STATE.  With the maps uploaded intact the same group solves
    again (the words were cleared when reported)."""
    from glide_b200 import _lib
    from glide_b200.group import HierarchyGroup
    members = _members(precision)[:3]
    g = HierarchyGroup([m.mg.hierarchy for m in members])
    g.set_tuning(spoil_maps=True)
    with pytest.raises(_lib.GlideError) as err:
        g.forward(DT)
    assert err.value.code == _lib.GLIDE_ERR_STATE
    assert "staging maps" in str(err.value)
    g.set_tuning(spoil_maps=False)
    for m in members:  # the state the failed call left is not a solve's; start again from the dome
        h = m.mg.hierarchy
        for f in ("u", "v"):
            h.set(f, 0, torch.zeros_like(h.get(f, 0)), restrict_down=True)
        h.set("H", 0, m.mg.levels[0].state.H_prev.data, restrict_down=True)
    st = g.forward(DT)
    assert all(np.isfinite(s["final_norm"]) and s["vcycles"] > 0 for s in st)
    g.close()


def test_group_reports_a_nonfinite_member_and_solves_the_others():
    """A member whose residual is not finite makes the group call return
    GLIDE_ERR_NONFINITE after the others finish; the others' solves are
    complete (they equal their solo solves), and the group stays usable."""
    from glide_b200 import _lib
    from glide_b200.group import HierarchyGroup
    solo, grouped = _members("fp64")[:3], _members("fp64")[:3]
    H = grouped[1].mg.hierarchy.get("H", 0).clone()
    H[5, 5] = float("nan")
    grouped[1].mg.hierarchy.set("H", 0, H, restrict_down=True)
    g = HierarchyGroup([m.mg.hierarchy for m in grouped])
    with pytest.raises(_lib.GlideError) as err:
        g.forward(DT)
    assert err.value.code == _lib.GLIDE_ERR_NONFINITE
    for k in (0, 2):
        solo[k].forward(0.0, DT, update_geometry=False)
        for f in ("u", "v", "H"):
            x = solo[k].mg.hierarchy.get(f, 0).cpu().numpy()
            y = grouped[k].mg.hierarchy.get(f, 0).cpu().numpy()
            assert rel_err(y, x) <= 1e-10, (k, f)
    # the non-finite member restored, the same group solves all three
    grouped[1].mg.hierarchy.set("H", 0, solo[1].mg.hierarchy.get("H", 0), restrict_down=True)
    st = g.forward(DT)
    assert all(np.isfinite(s["final_norm"]) for s in st)
    g.close()
