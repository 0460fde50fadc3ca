"""The oracle's coupled thermomechanical loop (oracle/coupled_oracle.py), on
the CPU, against the reference's own IceDynamics + ThermalModel run in the
same order (fixture tests/golden/coupled_f64.npz, made by
tests/golden/make_golden.py through oracle/refpy.py): three coupled steps on
a 32^2 x 9 dome, 2 V-cycles per momentum solve, at 1e-10."""
from __future__ import annotations

from util import load_golden, rel_err


def test_oracle_coupled_loop_matches_reference():
    from cases import dome
    from oracle.coupled_oracle import coupled_run
    g = load_golden("coupled_f64")
    f = dome(32, 48e3, 1200e3, seed=3)
    got = coupled_run(f, 48e3, 3, 9, 5.0, 3, 2)
    for k in ("u", "v", "H", "E", "B"):
        assert rel_err(got[k], g[f"out_{k}"]) <= 1e-10, (k, rel_err(got[k], g[f"out_{k}"]))
