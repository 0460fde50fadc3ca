"""Coupled thermomechanical steps (momentum + mass solve, then the enthalpy
column solve, B fed back) through the public API, in the order of the
reference's coupled example (examples/thermal/coupled_dome.py:258-272).

1. binary64, reference algorithm and quirks, fixed V-cycles: three coupled
   steps on a 32^2 x 9 dome against the oracle's coupled loop
   (oracle/coupled_oracle.py) and against the reference's own run of the
   same steps (tests/golden/coupled_f64.npz) at 1e-10 -- the multi-step
   drift of the B feedback and of omega from the realised dH/dt, checked.
2. the bench's fast form: five coupled steps on a 256^2 x 41 dome (the
   large run's recipe, coarser cells), mixed precision against binary64,
   both solved to a relative residual of 1e-8; the errors the mixed form
   makes against binary64 are asserted at the tolerances written below.
"""
from __future__ import annotations

import numpy as np
import pytest

from util import load_golden, rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_coupled_binary64_matches_oracle():
    from cases import CoupledRun, dome
    from oracle.coupled_oracle import coupled_run
    n, dx, levels, nz, steps, cycles = 32, 48e3, 3, 9, 3, 2
    f = dome(n, dx, 1200e3, seed=3)
    run = CoupledRun(f, dx, levels, nz, precision="fp64", quirks=True, rtol=0.0, max_vcycles=cycles)
    sweeps = []
    for _ in range(steps):
        st, sw = run.step()
        assert st["vcycles"] == cycles
        sweeps.append(sw)
    got = run.fields()
    ref = coupled_run(f, dx, levels, nz, 5.0, steps, cycles)
    assert sweeps == ref["sweeps"]
    g = load_golden("coupled_f64")  # the reference's own run of the same steps
    for k in ("u", "v", "H", "E", "B"):
        assert rel_err(got[k], ref[k]) <= 1e-10, k
        assert rel_err(got[k], g[f"out_{k}"]) <= 1e-10, k


# mixed (binary32 smoother and tangent multigrid, binary64 residual and
# state) against binary64 after five coupled steps, both to 1e-8.  Both end
# in Newton steps on the same binary64 residual, which overshoot the solve
# tolerance; measured differences are ~1e-14 (u, v) and ~1e-15 (H, E, B).
MIXED_TOL = {"u": 1e-8, "v": 1e-8, "H": 1e-9, "E": 1e-9, "B": 1e-9}


def test_coupled_mixed_matches_binary64():
    from cases import CoupledRun, configure_fast, dome
    n, dx, levels, nz, steps = 256, 6000.0, 4, 41, 5
    f = dome(n, dx, 1200e3, seed=0)
    out = {}
    for prec in ("mixed", "fp64"):
        run = CoupledRun(f, dx, levels, nz, precision=prec, quirks=False, configure=configure_fast, rtol=1e-8)
        rels = []
        for _ in range(steps):
            st, _ = run.step()
            rels.append(st["final_norm"] / st["initial_norm"])
        assert max(rels) <= 1e-8, (prec, rels)
        out[prec] = run.fields()
        del run
    errs = {k: rel_err(out["mixed"][k], out["fp64"][k]) for k in MIXED_TOL}
    print("coupled mixed vs binary64:", errs)
    for k, tol in MIXED_TOL.items():
        assert errs[k] <= tol, (k, errs[k])
