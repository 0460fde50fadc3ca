"""Ensemble of uneven members: member layout on the CPU, and on the GPU the
concurrent driver gives bit-identical results to running every member alone
(members are independent; streams and threads change no arithmetic)."""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_levels_for_reaches_coarsest_at_least_16():
    from glide_b200.ensemble import levels_for
    assert [levels_for(n) for n in (128, 192, 256, 384, 512, 768)] == [4, 4, 5, 5, 6, 6]
    for n in (128, 192, 256, 384, 512, 768):
        L = levels_for(n)
        assert n % 2 ** (L - 1) == 0 and n // 2 ** (L - 1) >= 16
        assert n % 2 ** L != 0 or n // 2 ** L < 16  # one more level would break the rule


def test_member_specs_are_seeded_and_uneven():
    from glide_b200.ensemble import member_specs
    a, b = member_specs(64, seed=3), member_specs(64, seed=3)
    assert a == b
    assert len({m.n for m in a}) >= 5
    for m in a:
        assert 0 < m.radius <= 600e3 and 1e-3 <= m.lapse <= 3e-3
        assert m.radius <= 0.45 * m.n * m.dx


def _member(n, seed, levels=3, dx=4000.0):
    from cases import dome
    from glide_b200.model import IceDynamics
    f = dome(n, dx, R=0.4 * n * dx, seed=seed)
    m = IceDynamics(n_levels=levels, ny=n, nx=n, dx=dx, reference_quirks=False)
    mg = m.mg
    for k, grp in (("bed", mg.geometry), ("B", mg.rheology), ("beta", mg.sliding), ("smb", mg.forcing)):
        getattr(grp, k).set(torch.as_tensor(f[k]))
    mg.state.H.set(torch.as_tensor(f["H"]))
    mg.state.H_prev.set(torch.as_tensor(f["H_prev"]))
    m.forward_solver.fas_options.set(maximum_vcycles=6, relative_tolerance=0.0, absolute_tolerance=0.0,
                                     report_norms=False)
    m.adjoint_solver.fas_options.set(maximum_vcycles=3, relative_tolerance=0.0, absolute_tolerance=0.0,
                                     report_norms=False)
    return m


@pytest.mark.gpu
def test_concurrent_members_match_solo_runs():
    from glide_b200.ensemble import Ensemble
    sizes = [64, 96, 128, 64, 96]

    def run(concurrent):
        members = [_member(n, seed=10 + k) for k, n in enumerate(sizes)]
        dJ = lambda k, m: (0.05 * m.mg.levels[0].state.u.data, 0.05 * m.mg.levels[0].state.v.data, None)
        if concurrent:
            ens = Ensemble(members, workers=3)
            for step in range(2):
                ens.forward(step * 10.0, 10.0, retry=False)
            ens.backward(20.0, 10.0, dJ)
            torch.cuda.synchronize()
            ens.close()
        else:
            for m in members:
                for step in range(2):
                    m.forward(step * 10.0, 10.0)
                du, dv, _ = dJ(0, m)
                m.backward(20.0, 10.0, dJdu=du, dJdv=dv)
            torch.cuda.synchronize()
        return [{k: m.mg.hierarchy.get(k, 0).cpu().numpy() for k in ("u", "v", "H", "lambda_u", "grad_beta")}
                for m in members]

    a, b = run(True), run(False)
    for ma, mb in zip(a, b):
        for k in ma:
            np.testing.assert_array_equal(ma[k], mb[k], err_msg=k)


@pytest.mark.gpu
def test_forward_retries_other_schedules_when_a_solve_stops_short():
    """A member whose solve stops at its cycle cap short of the tolerance is
    solved again under each other candidate schedule until one converges;
    with a one-cycle cap none does, so every other candidate is tried once
    and the member keeps its schedule."""
    from glide_b200.ensemble import CANDIDATES, FALLBACK, Ensemble, apply_schedule
    m = _member(64, seed=3)
    m.forward_solver.fas_options.set(maximum_vcycles=1, relative_tolerance=1e-12, absolute_tolerance=0.0)
    ens = Ensemble([m], workers=1)
    apply_schedule(m, CANDIDATES["fascd"])
    ens.schedules[0] = "fascd"
    st = ens.forward(0.0, 10.0)[0]
    torch.cuda.synchronize()
    ens.close()
    others = {n for n in list(CANDIDATES) + [FALLBACK] if n != "fascd"}
    assert ens.retries == len(others)
    assert ens.schedules[0] == "fascd"
    assert np.isfinite(st["final_norm"])
    H = m.mg.hierarchy.get("H", 0)
    assert bool(torch.equal(m.mg.hierarchy.get("H_prev", 0), H))


@pytest.mark.gpu
def test_grouped_ensemble_matches_solo_runs():
    """Grouped mode: the members of at most 96^2 cells solve in one grouped
    forward solve (FASCD and guarded Newton schedules) and one grouped
    adjoint solve while the 128^2 member solves on a worker stream; each
    member runs the cycles of its own solo solves and its fields agree with
    them to rounding (the grouped kernels are separate compilations of the
    same tile bodies)."""
    from util import rel_err
    from glide_b200.ensemble import CANDIDATES, Ensemble, apply_schedule
    sizes = [64, 96, 128, 64, 96]
    names = ["fast", "classic", "fast", "fascd/1", "newton/classic"]

    def build():
        members = [_member(n, seed=40 + k) for k, n in enumerate(sizes)]
        for m, name in zip(members, names):
            apply_schedule(m, CANDIDATES[name])
            m.forward_solver.fas_options.set(maximum_vcycles=30, relative_tolerance=1e-8)
            m.adjoint_solver.fas_options.set(maximum_vcycles=30, relative_tolerance=1e-8)
        return members

    dJ = lambda k, m: (0.05 * m.mg.levels[0].state.u.data, 0.05 * m.mg.levels[0].state.v.data, None)
    a, b = build(), build()
    ens = Ensemble(a, workers=2, grouped=True, group_max_cells=96 * 96)
    for k, name in enumerate(names):
        ens.schedules[k] = name
    fa = [ens.forward(step * 10.0, 10.0, retry=False) for step in range(2)]
    ba = ens.backward(20.0, 10.0, dJ)
    torch.cuda.synchronize()
    assert ens._fwd_keys == (0, 1, 3, 4) and ens._adj_keys == (0, 1, 3, 4)
    ens.close()
    fb = [[m.forward(step * 10.0, 10.0) for m in b] for step in range(2)]
    bb = []
    for k, m in enumerate(b):
        du, dv, _ = dJ(k, m)
        bb.append(m.backward(20.0, 10.0, dJdu=du, dJdv=dv))
    torch.cuda.synchronize()
    assert [[s["vcycles"] for s in f] for f in fa] == [[s["vcycles"] for s in f] for f in fb]
    assert [s["vcycles"] for s in ba] == [s["vcycles"] for s in bb]
    for ma, mb in zip(a, b):
        for k in ("u", "v", "H", "H_prev", "lambda_u", "lambda_H", "grad_beta", "grad_bed"):
            x, y = ma.mg.hierarchy.get(k, 0).cpu().numpy(), mb.mg.hierarchy.get(k, 0).cpu().numpy()
            assert rel_err(x, y) <= 1e-10, (k, rel_err(x, y))


def test_grouping_partitions_members_by_size_and_count():
    """Grouped mode's partition of the group members: one group per grid size
    (members in order), split into groups of at most `group_size`; "all"
    puts every member in one group before the split."""
    from types import SimpleNamespace
    from glide_b200.ensemble import Ensemble

    def fake(n):
        h = SimpleNamespace(shapes=[(n, n, 1500.0)], precision="fp64")
        return SimpleNamespace(mg=SimpleNamespace(hierarchy=h), top_level=0)

    sizes = [128, 256, 128, 768, 256, 128, 128]
    ens = Ensemble([fake(n) for n in sizes], workers=2, grouped=True)
    keys = tuple(range(len(sizes)))
    assert ens._parts(keys) == [(0, 2, 5, 6), (1, 4), (3,)]
    ens.group_size = 3
    assert ens._parts(keys) == [(0, 2, 5), (6,), (1, 4), (3,)]
    ens.group_by, ens.group_size = "all", 4
    assert ens._parts(keys) == [(0, 1, 2, 3), (4, 5, 6)]
    assert ens._parts(()) == []
    ens.group_max_cells = 256 * 256
    assert [k for k in keys if ens._in_groups(k)] == [0, 1, 2, 4, 5, 6]
    ens.members[1].mg.hierarchy.precision = "mixed"  # no grouped form: solved on the worker streams
    assert [k for k in keys if ens._in_groups(k)] == [0, 2, 4, 5, 6]
    ens.close()


def test_bench_ensemble_precision_defaults():
    """The bench's ensemble runs mixed-precision members by default, binary64
    members when grouped, and refuses grouped mixed members before it builds
    any member."""
    import bench
    a = bench.parse(["--mode", "ensemble", "--ens-grouped", "--ens-precision", "mixed"])
    with pytest.raises(SystemExit, match="grouped solves"):
        bench.run_ensemble(a)
    assert bench.parse(["--mode", "ensemble"]).ens_precision is None
