"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference package (JacobDowns/glide, read from its checkout) on host
cores through oracle/refpy.py: the reference's own Python sequencing, option
objects and CUDA kernel sources, the kernels executed by the host fiber
emulator.  binary64 fixtures use the binary64 build of the same sources; one
binary32 fixture uses the kernels as written.

    python tests/golden/make_golden.py [--reference DIR]

Each .npz stores the inputs it was made from and the reference's outputs.
"""
from __future__ import annotations

import argparse
import contextlib
import io
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

from cases import SEC_PER_YR, enthalpy_config, enthalpy_state, random_state, slab_c1  # noqa: E402
from oracle.refpy import load_reference  # noqa: E402


def quiet():
    return contextlib.redirect_stdout(io.StringIO())


def c1_forward_and_adjoint(glide, tag):
    from glide.model import IceDynamics
    f = slab_c1()
    with quiet():
        model = IceDynamics(n_levels=4, ny=64, nx=64, dx=1000.0)
    mg = model.mg
    for k in ("bed", "B", "beta", "smb"):
        getattr({"bed": mg.geometry, "B": mg.rheology, "beta": mg.sliding, "smb": mg.forcing}[k], k).set(f[k])
    mg.state.H.set(f["H"])
    mg.state.H_prev.set(f["H_prev"])
    s = model.forward_solver
    s.fas_options.set(maximum_vcycles=3, relative_tolerance=0.0, absolute_tolerance=0.0, report_norms=False)
    with quiet():
        model.forward(0.0, 10.0, update_geometry=False)
    lv = mg.levels[0]
    out = {f"in_{k}": np.asarray(v) for k, v in f.items()}
    for k in ("u", "v", "H", "mask", "phi"):
        out[f"out_{k}"] = np.array(getattr(lv.state, k).data, dtype=np.float64)
    np.savez_compressed(HERE / f"c1_forward_{tag}.npz", **out)
    if tag != "f64":
        return
    u, v = np.array(lv.state.u.data), np.array(lv.state.v.data)
    dJdu = u - 1.1 * u
    dJdv = v - 0.9 * v
    a = model.adjoint_solver
    a.fas_options.set(maximum_vcycles=2, relative_tolerance=0.0, absolute_tolerance=0.0, report_norms=False)
    with quiet():
        model.backward(0.0, 10.0, dJdu=dJdu, dJdv=dJdv)
    adj = dict(out)
    adj["in_dJdu"], adj["in_dJdv"] = dJdu, dJdv
    for k in ("lambda_u", "lambda_v", "lambda_H"):
        adj[f"out_{k}"] = np.array(getattr(lv.adjoint, k).data)
    adj["out_grad_beta"] = np.array(lv.sliding.beta.grad)
    adj["out_grad_bed"] = np.array(lv.geometry.bed.grad)
    adj["out_grad_H_prev"] = np.array(lv.state.H_prev.grad)
    adj["out_grad_smb"] = np.array(lv.forcing.smb.grad)
    np.savez_compressed(HERE / "c1_adjoint_f64.npz", **adj)


def random_grid(glide, st, calving=0.0):
    from glide.grid import Grid
    ny, nx = st["H"].shape
    g = Grid(ny, nx, 1500.0)
    for k in ("u", "v", "H", "H_prev", "mask"):
        getattr(g.state, k).set(st[k])
    g.geometry.bed.set(st["bed"])
    g.rheology.B.set(st["B"])
    g.sliding.beta.set(st["beta"])
    g.forcing.smb.set(st["smb"])
    g.calving.calving_rate.set(calving)
    g.forward_operators.f_u[:, :] = st["f_u"]
    g.forward_operators.f_v[:, :] = st["f_v"]
    return g


def random_cases(glide):
    st = random_state(40, 56, seed=7)
    dt = 5.0
    out = {f"in_{k}": v for k, v in st.items()}
    for tag, calving in (("", 0.0), ("_calving", 2.0)):
        g = random_grid(glide, st, calving)
        ops = g.forward_operators
        ops.set_rhs(dt)
        ops.compute_residual(dt, use_mask=True)
        for k in ("r_u", "r_v", "r_H"):
            out[f"out_{k}{tag}"] = np.array(getattr(ops, k))
        out[f"out_phi{tag}"] = np.array(g.state.phi.data)
        ops.compute_residual(dt, use_mask=False, operator_only=True, freeze_phi=True)
        for k in ("F_u", "F_v", "F_H"):
            out[f"out_{k}{tag}"] = np.array(getattr(ops, k))
    np.savez_compressed(HERE / "random_residual_f64.npz", **out)

    out = {f"in_{k}": v for k, v in st.items()}
    g = random_grid(glide, st)
    ops = g.forward_operators
    ops.set_rhs(dt)
    ops.vanka_sweep(dt, 3)
    for k in ("u", "v", "H", "mask", "phi"):
        out[f"out_{k}"] = np.array(getattr(g.state, k).data)
    np.savez_compressed(HERE / "random_vanka_f64.npz", **out)

    # forward-mode derivative (ForwardOperators.compute_jvp)
    rng = np.random.default_rng(5)
    ny, nx = st["H"].shape
    var = dict(var_u=rng.normal(0, 1, (ny, nx + 1)), var_v=rng.normal(0, 1, (ny + 1, nx)),
               var_H=rng.normal(0, 10, (ny, nx)))
    out = {f"in_{k}": v for k, v in {**st, **var}.items()}
    g = random_grid(glide, st)
    ops = g.forward_operators
    ops.set_rhs(dt)
    for k, v in var.items():
        getattr(ops, k)[:, :] = v
    ops.compute_jvp(dt)
    for k in ("jvp_u", "jvp_v", "jvp_H"):
        out[f"out_{k}"] = np.array(getattr(ops, k))
    out["out_phi"] = np.array(g.state.phi.data)
    np.savez_compressed(HERE / "random_jvp_f64.npz", **out)

    rng = np.random.default_rng(11)
    ny, nx = st["H"].shape
    lam = dict(lambda_u=rng.normal(0, 1, (ny, nx + 1)), lambda_v=rng.normal(0, 1, (ny + 1, nx)),
               lambda_H=rng.normal(0, 1, (ny, nx)))
    af = dict(adj_f_u=rng.normal(0, 1, (ny, nx + 1)), adj_f_v=rng.normal(0, 1, (ny + 1, nx)),
              adj_f_H=rng.normal(0, 1, (ny, nx)))
    out = {f"in_{k}": v for k, v in {**st, **lam, **af}.items()}
    g = random_grid(glide, st)
    g.forward_operators.compute_phi()
    for k, v in lam.items():
        getattr(g.adjoint, k).set(v)
    aops = g.adjoint_operators
    aops.f_u[:, :] = af["adj_f_u"]
    aops.f_v[:, :] = af["adj_f_v"]
    aops.f_H[:, :] = af["adj_f_H"]
    aops.compute_vjp(dt)
    for k in ("vjp_u", "vjp_v", "vjp_H"):
        out[f"out_{k}"] = np.array(getattr(aops, k))
    aops.compute_residual(dt)
    for k in ("r_u", "r_v", "r_H"):
        out[f"out_adj_{k}"] = np.array(getattr(aops, k))
    aops.vanka_sweep(dt, 2)
    for k in ("lambda_u", "lambda_v", "lambda_H"):
        out[f"out_sweep_{k}"] = np.array(getattr(g.adjoint, k).data)
    aops.compute_gradient_beta()
    aops.compute_gradient_bed()
    out["out_grad_beta"] = np.array(g.sliding.beta.grad)
    out["out_grad_bed"] = np.array(g.geometry.bed.grad)
    out["out_phi"] = np.array(g.state.phi.data)
    np.savez_compressed(HERE / "random_adjoint_f64.npz", **out)


def jvp_flag_cases(glide):
    """ForwardOperators.compute_jvp (glide/operators.py:129-171) with its
    use_mask and freeze_calving flags on the random state with a calving rate
    of 2: the default flags, use_mask=False, and freeze_calving=True."""
    st = random_state(40, 56, seed=7)
    dt = 5.0
    rng = np.random.default_rng(5)
    ny, nx = st["H"].shape
    var = dict(var_u=rng.normal(0, 1, (ny, nx + 1)), var_v=rng.normal(0, 1, (ny + 1, nx)),
               var_H=rng.normal(0, 10, (ny, nx)))
    out = {f"in_{k}": v for k, v in {**st, **var}.items()}
    out["in_calving_rate"] = np.array(2.0)
    for tag, kw in (("", {}), ("_nomask", dict(use_mask=False)), ("_frozen", dict(freeze_calving=True))):
        g = random_grid(glide, st, calving=2.0)
        ops = g.forward_operators
        ops.set_rhs(dt)
        for k, v in var.items():
            getattr(ops, k)[:, :] = v
        ops.compute_jvp(dt, **kw)
        for k in ("jvp_u", "jvp_v", "jvp_H"):
            out[f"out_{k}{tag}"] = np.array(getattr(ops, k))
    np.savez_compressed(HERE / "random_jvp_flags_f64.npz", **out)


def coupled_case(glide):
    """Three coupled thermomechanical steps with the reference's own
    IceDynamics and ThermalModel, in the order of its coupled example
    (examples/thermal/coupled_dome.py:258-272): a 32^2 dome (dx 48 km, R =
    1200 km, seed 3), 3 levels, 9 sigma levels, dt 5 a, each momentum solve 2
    FASCD V-cycles, surface temperature -30 + 6e-3 (2000 - s) C, geothermal
    flux 0.05 W m^-2, B first set from the initial temperature on every level
    (coupled_dome.py:144-146)."""
    from glide.model import IceDynamics, ThermalModel
    from cases import dome, surface_temperature
    n, dx, levels, nz, steps, dt_yr = 32, 48e3, 3, 9, 3, 5.0
    f = dome(n, dx, 1200e3, seed=3)
    with quiet():
        model = IceDynamics(n_levels=levels, ny=n, nx=n, dx=dx)
    mg = model.mg
    for k, grp in (("bed", mg.geometry), ("B", mg.rheology), ("beta", mg.sliding), ("smb", mg.forcing)):
        getattr(grp, k).set(f[k])
    mg.state.H.set(f["H"])
    mg.state.H_prev.set(f["H_prev"])
    model.forward_solver.fas_options.set(maximum_vcycles=2, relative_tolerance=0.0, absolute_tolerance=0.0,
                                         report_norms=False)
    grid = mg.levels[0]
    tm = ThermalModel(grid, nz=nz, n_smooth=10)
    tm.initialize(surface_temperature(np.array(grid.state.H.data), np.array(grid.geometry.bed.data)), Q_geo=0.05)
    mg.rheology.B.set(tm.ops.get_arrhenius_factor() / tm.B_scale)
    for _ in range(steps):
        tm.pre_momentum()
        with quiet():
            model.forward(0.0, dt_yr)
        tm.ops.set_surface_enthalpy_from_temperature(
            surface_temperature(np.array(grid.state.H.data), np.array(grid.geometry.bed.data)))
        tm.step(dt_yr * SEC_PER_YR)
    out = {"out_u": np.array(grid.state.u.data), "out_v": np.array(grid.state.v.data),
           "out_H": np.array(grid.state.H.data), "out_E": np.array(tm.enthalpy),
           "out_B": np.array(grid.rheology.B.data)}
    np.savez_compressed(HERE / "coupled_f64.npz", **out)


C3_STRIDE = 7  # the sampling lattice of the 512^2 fixture (prime: not aligned with any tile)


def c3_dome_case(glide):
    """The C3 dome at full size: 512^2, dx 1500 m, 5 levels, dt 10 a, the
    reference algorithm (its defaults and quirks), 3 forward V-cycles, then
    the adjoint of dJ/du = 0.05 u, dJ/dv = 0.05 v with 2 V-cycles and the
    gradients.  Inputs are regenerated by tests/cases.py dome(512, 1500,
    600e3, seed=0); the fixture keeps their checksums, every field's
    max-norm and its values on a stride-7 lattice."""
    from glide.model import IceDynamics
    from cases import dome
    f = dome(512, 1500.0, 600e3, seed=0)
    with quiet():
        model = IceDynamics(n_levels=5, ny=512, nx=512, dx=1500.0)
    mg = model.mg
    for k, grp in (("bed", mg.geometry), ("B", mg.rheology), ("beta", mg.sliding), ("smb", mg.forcing)):
        getattr(grp, k).set(f[k])
    mg.state.H.set(f["H"])
    mg.state.H_prev.set(f["H_prev"])
    model.forward_solver.fas_options.set(maximum_vcycles=3, relative_tolerance=0.0, absolute_tolerance=0.0,
                                         report_norms=False)
    with quiet():
        model.forward(0.0, 10.0, update_geometry=False)
    lv = mg.levels[0]
    u, v = np.array(lv.state.u.data), np.array(lv.state.v.data)
    model.adjoint_solver.fas_options.set(maximum_vcycles=2, relative_tolerance=0.0, absolute_tolerance=0.0,
                                         report_norms=False)
    with quiet():
        model.backward(0.0, 10.0, dJdu=0.05 * u, dJdv=0.05 * v)
    fields = {"u": lv.state.u.data, "v": lv.state.v.data, "H": lv.state.H.data,
              "lambda_u": lv.adjoint.lambda_u.data, "lambda_v": lv.adjoint.lambda_v.data,
              "lambda_H": lv.adjoint.lambda_H.data, "grad_beta": lv.sliding.beta.grad,
              "grad_bed": lv.geometry.bed.grad}
    out = {f"in_sum_{k}": np.array([float(np.sum(f[k])), float(np.sum(np.abs(f[k])))])
           for k in ("bed", "B", "beta", "smb", "H")}
    for k, a in fields.items():
        a = np.array(a, dtype=np.float64)
        out[f"max_{k}"] = np.array(float(np.abs(a).max()))
        out[f"out_{k}"] = a[::C3_STRIDE, ::C3_STRIDE].copy()
    np.savez_compressed(HERE / "c3_dome512_f64.npz", **out)


def vanka_dump_case(glide):
    """ForwardOperators.vanka_dump (glide/operators.py:253-273) on the random
    state: the local 5x5 systems of every cell."""
    st = random_state(40, 56, seed=7)
    dt = 5.0
    g = random_grid(glide, st, calving=1.0)
    ops = g.forward_operators
    ops.set_rhs(dt)
    ops.compute_phi()
    J, r = ops.vanka_dump(dt)
    out = {f"in_{k}": v for k, v in st.items()}
    out["in_phi"] = np.array(g.state.phi.data)
    out["in_gamma"] = np.array(ops.gamma)
    out["out_J"] = np.array(J)
    out["out_r"] = np.array(r)
    np.savez_compressed(HERE / "random_vanka_dump_f64.npz", **out)


def transfer_cases(glide):
    """Multigrid.restrict_* / prolongate_* (glide/multigrid.py:118-259) on
    seeded arrays: every method on a square 16 x 16 grid (prolongate_hfacet is
    the reference's u-face kernel run on v arrays), and all but
    prolongate_hfacet on a 12 x 20 grid.  The reference's own v-face
    prolongation kernels, which its Python never launches, are run directly
    (transfer.cu:232-323)."""
    with quiet():
        mg = glide.multigrid.Multigrid(n_levels=2, ny=16, nx=16, dx=1000.0)
    rng = np.random.default_rng(11)
    out = {}
    for tag, (ny, nx) in (("sq", (16, 16)), ("rect", (12, 20))):
        nyc, nxc = ny // 2, nx // 2
        fine = {"u": rng.standard_normal((ny, nx + 1)), "v": rng.standard_normal((ny + 1, nx)),
                "c": rng.standard_normal((ny, nx))}
        coarse = {"u": rng.standard_normal((nyc, nxc + 1)), "v": rng.standard_normal((nyc + 1, nxc)),
                  "c": rng.standard_normal((nyc, nxc))}
        for k, v in fine.items():
            out[f"{tag}_fine_{k}"] = v
        for k, v in coarse.items():
            out[f"{tag}_coarse_{k}"] = v
        out[f"{tag}_restrict_vfacet"] = np.array(mg.restrict_vfacet(fine["u"]))
        out[f"{tag}_restrict_hfacet"] = np.array(mg.restrict_hfacet(fine["v"]))
        for m in ("avg", "max", "min", "var"):
            out[f"{tag}_restrict_cell_{m}"] = np.array(mg.restrict_cell(fine["c"], method=m))
        for m in ("injection", "bilinear"):
            out[f"{tag}_prolongate_vfacet_{m}"] = np.array(mg.prolongate_vfacet(coarse["u"], method=m))
            out[f"{tag}_prolongate_cell_{m}"] = np.array(mg.prolongate_cell(coarse["c"], method=m))
            if ny == nx:
                out[f"{tag}_prolongate_hfacet_{m}"] = np.array(mg.prolongate_hfacet(coarse["v"], method=m))
            f = np.zeros((ny + 1, nx))
            n = (ny + 1) * nx
            glide._kernels.launch(f"prolongate_hfacet_{m}", (n + 255) // 256, 256, (coarse["v"], f, ny, nx))
            out[f"{tag}_vface_prolongate_hfacet_{m}"] = f
    np.savez_compressed(HERE / "transfers_f64.npz", **out)


def enthalpy_cases(glide):
    """EnthalpyOperators (glide/enthalpy.py) on a rough random state: residual,
    one column smooth, one layer smooth, omega, and column sweeps; then one
    ThermalModel step (glide/model.py:97-281) on a random grid."""
    from glide.enthalpy import EnthalpyOperators
    from glide.grid import Grid
    from glide.model import ThermalModel
    ny, nx, nz = 6, 9, 11
    st = enthalpy_state(ny, nx, nz, seed=5)
    cfg = enthalpy_config()
    dt = cfg["dt"]

    def make_ops():
        g = Grid(ny, nx, cfg["dx"])
        g.state.H.set(st["H"])
        ops = EnthalpyOperators(g, nz=nz)
        es, ev, ef = ops.enthalpy_state, ops.enthalpy_velocity, ops.enthalpy_forcing
        es.E[:] = st["E"]
        es.E_prev[:] = st["E_prev"]
        ops.f_E[:] = st["f_E"]
        ev.u3d[:] = st["u3d"]
        ev.v3d[:] = st["v3d"]
        ev.omega[:] = st["omega"]
        ops.H_prev[:] = st["H_prev"]
        ef.E_surface[:] = st["E_surface"]
        return ops

    out = {f"in_{k}": v for k, v in st.items()}
    ops = make_ops()
    out["out_rmax"] = np.array(ops.compute_residual(dt))
    out["out_r_E"] = np.array(ops.r_E)
    ops.column_smooth(dt)
    out["out_column_delta"] = np.array(ops.delta_E)
    ops.layer_smooth(dt)
    out["out_layer_delta"] = np.array(ops.delta_E)
    rng = np.random.default_rng(17)
    dh = rng.normal(0.0, 0.5, (ny, nx))
    out["in_dh_dt"] = dh
    ev = ops.enthalpy_velocity
    ev.u3d[:] = st["u3d"] * SEC_PER_YR
    ev.v3d[:] = st["v3d"] * SEC_PER_YR
    ops.compute_omega(dh)
    out["out_omega"] = np.array(ev.omega)
    for tag, alternating, n in (("alt", True, 4), ("col", False, 3)):
        ops = make_ops()
        ops.smoother_config.relative_tolerance = 1e-30
        ops.smoother_config.absolute_tolerance = 0.0
        ops.column_sweep(dt, n, alternating=alternating)
        out[f"out_sweep_{tag}_E"] = np.array(ops.enthalpy_state.E)
    np.savez_compressed(HERE / "enthalpy_ops_f64.npz", **out)

    # one coupled thermal step
    ny, nx, nz = 8, 10, 9
    rng = np.random.default_rng(23)
    g = Grid(ny, nx, 1500.0)
    u = rng.normal(0.0, 80.0, (ny, nx + 1))
    v = rng.normal(0.0, 80.0, (ny + 1, nx))
    H0 = rng.uniform(200.0, 2500.0, (ny, nx))
    H0[0, :3] = 10.0
    beta = rng.uniform(0.05, 0.5, (ny, nx))
    T_s = rng.uniform(238.0, 268.0, (ny, nx))
    g.state.u.set(u)
    g.state.v.set(v)
    g.state.H.set(H0)
    g.sliding.beta.set(beta)
    tm = ThermalModel(g, nz=nz, n_smooth=4)
    tm.initialize(T_s, Q_geo=0.05)
    tm.pre_momentum()
    H1 = H0 * rng.uniform(0.99, 1.01, (ny, nx))
    g.state.H.set(H1)
    dt_s = 10.0 * SEC_PER_YR
    tm.step(dt_s)
    out = dict(in_u=u, in_v=v, in_H0=H0, in_H1=H1, in_beta=beta, in_T_s=T_s, in_dt=np.array(dt_s))
    out["out_E"] = np.array(tm.enthalpy)
    out["out_omega"] = np.array(tm.ops.enthalpy_velocity.omega)
    out["out_Q_fh"] = np.array(tm.ops.enthalpy_forcing.Q_fh)
    out["out_B"] = np.array(g.rheology.B.data)
    out["out_T"] = np.array(tm.temperature)
    np.savez_compressed(HERE / "thermal_step_f64.npz", **out)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--only", default=None,
                    help="enthalpy | dump | transfers | jvp_flags | c3 | coupled: only those fixtures")
    a = ap.parse_args(argv)
    if a.only == "coupled":
        coupled_case(load_reference(fp64=True, reference=a.reference))
        return
    if a.only == "c3":
        c3_dome_case(load_reference(fp64=True, reference=a.reference))
        return
    if a.only == "jvp_flags":
        jvp_flag_cases(load_reference(fp64=True, reference=a.reference))
        return
    if a.only == "enthalpy":
        enthalpy_cases(load_reference(fp64=True, reference=a.reference))
        return
    if a.only == "dump":
        vanka_dump_case(load_reference(fp64=True, reference=a.reference))
        return
    if a.only == "transfers":
        transfer_cases(load_reference(fp64=True, reference=a.reference))
        return
    glide = load_reference(fp64=True, reference=a.reference)
    c1_forward_and_adjoint(glide, "f64")
    random_cases(glide)
    jvp_flag_cases(glide)
    enthalpy_cases(glide)
    vanka_dump_case(glide)
    transfer_cases(glide)
    c3_dome_case(glide)
    coupled_case(glide)
    glide32 = load_reference(fp64=False, reference=a.reference)
    c1_forward_and_adjoint(glide32, "f32")
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
