"""Seeded synthetic inputs with the shapes and value ranges of the workloads
(no datasets exist here; these stand in for them).

* `slab_c1`   -- 64x64, dx = 1 km, 4 levels, dt = 10 a: tilted bed with a
                 500 m sinusoidal bump, uniform 1000 m ice, A = 1e-16, beta
                 1000 + 500 sin(2 pi x / 64 km) (ISMIP-HOM-like slab).
* `dome`      -- radius-R Vialov-style dome, H = 3000 (1 - (r/R)^(4/3))^(3/8)
                 floored at 0.1 m, Gaussian random bed (spectral slope -3,
                 std 400 m, mean 200 m), log-normal beta smoothed over 10 km,
                 smb = 0.5 - 2e-3 (s - 1500), A = 1e-16.
All parameters are in the reference's "head units": B and beta divided by
rho_i g with rho_i = 910 kg m^-3, g = 9.81 m s^-2.
"""
from __future__ import annotations

import numpy as np

RHO_I = 910.0
G = 9.81


def slab_c1(ny=64, nx=64, dx=1000.0):
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    X, Y = np.meshgrid(x, y)
    L = 64e3
    bed = -X * np.tan(np.deg2rad(0.5)) + 500.0 * np.sin(2 * np.pi * X / L) * np.sin(2 * np.pi * Y / L)
    H = np.full((ny, nx), 1000.0)
    B = np.full((ny, nx), (1e-16 ** (-1.0 / 3.0)) / (RHO_I * G))
    beta = (1000.0 + 500.0 * np.sin(2 * np.pi * X / L)) / (RHO_I * G)
    smb = np.full((ny, nx), 0.3)
    return dict(bed=bed, H=H, H_prev=H.copy(), B=B, beta=beta, smb=smb)


def _smooth(field, sigma_cells):
    """Gaussian smoothing by FFT (periodic), width in cells."""
    ny, nx = field.shape
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    g = np.exp(-2 * (np.pi * sigma_cells) ** 2 * (kx ** 2 + ky ** 2))
    return np.fft.ifft2(np.fft.fft2(field) * g).real


def dome(n=512, dx=1500.0, R=600e3, seed=0, lapse=2e-3):
    rng = np.random.default_rng(seed)
    c = (np.arange(n) + 0.5) * dx - n * dx / 2
    X, Y = np.meshgrid(c, c)
    r = np.sqrt(X ** 2 + Y ** 2)
    H = 3000.0 * np.clip(1.0 - (r / R) ** (4.0 / 3.0), 0.0, None) ** (3.0 / 8.0)
    H = np.maximum(H, 0.1)
    k = np.sqrt(np.fft.fftfreq(n)[:, None] ** 2 + np.fft.fftfreq(n)[None, :] ** 2)
    k[0, 0] = 1.0
    w = np.fft.ifft2(np.fft.fft2(rng.standard_normal((n, n))) * k ** (-1.5)).real
    bed = 200.0 + 400.0 * (w - w.mean()) / w.std()
    beta = np.exp(rng.normal(np.log(2000.0), 0.8, (n, n)))
    beta = _smooth(beta, 10e3 / dx) / (RHO_I * G)
    s = np.maximum(bed + H, (1.0 - 0.917) * H)
    smb = 0.5 - lapse * (s - 1500.0)
    B = np.full((n, n), (1e-16 ** (-1.0 / 3.0)) / (RHO_I * G))
    return dict(bed=bed, H=H, H_prev=H.copy(), B=B, beta=beta, smb=smb)


def random_state(ny, nx, seed=1, thin_frac=0.2):
    """A rough state exercising every branch: random velocities, thickness
    with thin-ice patches at the floor, mixed grounding, random mask."""
    rng = np.random.default_rng(seed)
    u = rng.normal(0, 50, (ny, nx + 1))
    v = rng.normal(0, 50, (ny + 1, nx))
    H = rng.uniform(50, 1500, (ny, nx))
    H[rng.random((ny, nx)) < thin_frac] = 0.1
    bed = rng.normal(-200, 400, (ny, nx))
    B = np.full((ny, nx), (1e-16 ** (-1.0 / 3.0)) / (RHO_I * G)) * rng.uniform(0.8, 1.2, (ny, nx))
    beta = rng.uniform(0.05, 0.5, (ny, nx))
    smb = rng.normal(0.3, 0.5, (ny, nx))
    mask = (rng.random((ny, nx)) < 0.15).astype(float)
    f_u = rng.normal(0, 1e-2, (ny, nx + 1))
    f_v = rng.normal(0, 1e-2, (ny + 1, nx))
    H_prev = H * rng.uniform(0.95, 1.05, (ny, nx))
    return dict(u=u, v=v, H=H, H_prev=H_prev, bed=bed, B=B, beta=beta, smb=smb, mask=mask, f_u=f_u, f_v=f_v)


SEC_PER_YR = 365.25 * 86400.0
E_SCALE_HOST = 2009.0 * (273.15 - 223.15)  # C_I (T_MELT - T_REF), J/kg


def enthalpy_state(ny, nx, nz, seed=1, thin_frac=0.15):
    """A rough enthalpy state exercising every branch of the column solver:
    cold and temperate nodes on both sides of the pressure-melting point,
    thin columns below h_thin, random layer velocities (m/s) and omega."""
    rng = np.random.default_rng(seed)
    H = rng.uniform(100.0, 3000.0, (ny, nx))
    H[rng.random((ny, nx)) < thin_frac] = rng.uniform(1.0, 20.0)
    sigma = np.linspace(0.0, 1.0, nz)
    depth = (1.0 - sigma)[None, None, :] * H[:, :, None]
    E_pmp = 2009.0 * (273.15 - 7.9e-8 * 910.0 * 9.81 * depth - 223.15) / E_SCALE_HOST
    # offsets from -0.5 (cold) to +0.02 (temperate, ~2 kJ/kg above pmp)
    E = E_pmp + rng.uniform(-0.5, 0.02, (ny, nx, nz))
    E_prev = E + rng.normal(0.0, 0.01, E.shape)
    u3d = rng.normal(0.0, 100.0, (nz, ny, nx + 1)) / SEC_PER_YR
    v3d = rng.normal(0.0, 100.0, (nz, ny + 1, nx)) / SEC_PER_YR
    omega = rng.normal(0.0, 0.3, (ny, nx, nz)) / SEC_PER_YR
    f_E = rng.normal(0.0, 1e-6, (ny, nx, nz))
    f_E[:, :, -1] = 0.0
    E_surface = E_pmp[:, :, -1] - rng.uniform(0.1, 0.4, (ny, nx))
    H_prev = H * rng.uniform(0.98, 1.02, (ny, nx))
    return dict(E=E, E_prev=E_prev, f_E=f_E, u3d=u3d, v3d=v3d, omega=omega, H=H, H_prev=H_prev,
                E_surface=E_surface)


def enthalpy_config(**kw):
    """ColumnSmootherConfig / EnthalpyForcing defaults of the reference
    (glide/enthalpy.py:108-203) as binary64 numbers."""
    cfg = dict(dx=2000.0, dt=10.0 * SEC_PER_YR, drain_rate=0.01 / SEC_PER_YR, h_thin=25.0,
               lf_c=1e-12, term_flags=7, omega=1.0, n_newton=3, relaxation=1.0,
               relative_tolerance=1e-5, absolute_tolerance=1e-2)
    cfg.update(kw)
    return cfg


def surface_temperature(H, bed):
    """The large thermomechanical run's surface temperature in K:
    -30 + 6e-3 (2000 - s) C with s = max(bed + H, (1 - 0.917) H).  Works on
    torch tensors and NumPy arrays alike (same operations in the same order)."""
    if isinstance(H, np.ndarray):
        s = np.maximum(bed + H, (1.0 - 0.917) * H)
    else:
        import torch
        s = torch.maximum(bed + H, (1.0 - 0.917) * H)
    return 273.15 + (-30.0 + 6e-3 * (2000.0 - s))


def configure_fast(h, mixed_inner=2):
    """The bench's fast solver form on a Hierarchy handle: corrected
    transfers, FASCD 4/4/0/50 with the local Newton capped at 3 iterations,
    guarded Newton from the first cycle with a 4/4/0/10 tangent multigrid."""
    h.set_reference_quirks(False)
    h.set_fas(False, pre_steps=4, post_steps=4, finest_steps=0, coarsest_steps=50)
    h.set_vanka(False, -1, newton_steps=3)
    h.set_tuning(forward_method="newton", newton_switch_exp10=0, mixed_inner_vcycles=mixed_inner)
    h.set_fas(2, pre_steps=4, post_steps=4, finest_steps=0, coarsest_steps=10)


class CoupledRun:
    """Coupled thermomechanical time steps through the public API, in the
    order of the reference's coupled example
    (examples/thermal/coupled_dome.py:258-272): ThermalModel.pre_momentum,
    IceDynamics.forward, the surface enthalpy from the new geometry,
    ThermalModel.step (which feeds B back into the finest grid).

    f: dome fields; precision "fp64" or "mixed" for the momentum solve (the
    enthalpy solve is binary64 either way); configure(h) sets solver options
    on the model's Hierarchy handle (None keeps the reference's algorithm).
    init_B: start from the rate factor of the initial temperature on every
    level (f's B is used only when False)."""

    def __init__(self, f, dx, n_levels, nz, precision="fp64", quirks=True, configure=None, rtol=1e-8,
                 max_vcycles=40, dt_yr=5.0, n_smooth=10, Q_geo=0.05, init_B=True):
        import torch
        from glide_b200.model import IceDynamics, ThermalModel
        ny, nx = f["H"].shape
        self.model = IceDynamics(n_levels=n_levels, ny=ny, nx=nx, dx=dx, reference_quirks=quirks,
                                 precision=precision)
        mg = self.model.mg
        for k, grp in (("bed", mg.geometry), ("B", mg.rheology), ("beta", mg.sliding), ("smb", mg.forcing)):
            getattr(grp, k).set(torch.as_tensor(f[k]))
        mg.state.H.set(torch.as_tensor(f["H"]))
        mg.state.H_prev.set(torch.as_tensor(f["H_prev"]))
        self.model.forward_solver.fas_options.set(maximum_vcycles=max_vcycles, relative_tolerance=rtol,
                                                  absolute_tolerance=0.0, report_norms=False)
        if configure is not None:
            configure(mg.hierarchy)
        self.grid = mg.levels[0]
        self.thermal = ThermalModel(self.grid, nz=nz, n_smooth=n_smooth)
        self.thermal.initialize(self.surface_T(), Q_geo=Q_geo)
        if init_B:
            # B from the initial temperature on every level, as the
            # reference's coupled example starts (coupled_dome.py:144-146)
            tm = self.thermal
            mg.rheology.B.set(tm.ops.get_arrhenius_factor(scale=tm.B_scale))
        self.dt_yr = dt_yr
        self.dt_s = dt_yr * SEC_PER_YR
        self.t = 0.0

    def surface_T(self):
        return surface_temperature(self.grid.state.H.data, self.grid.geometry.bed.data)

    def step(self, marks=None):
        """One coupled step; returns the momentum solve's stats and the
        number of enthalpy column sweeps it took.  marks: optional list of
        three CUDA events, recorded before the momentum solve, between it and
        the thermal half, and at the end."""
        tm = self.thermal
        if marks:
            marks[0].record()
        tm.pre_momentum()
        st = self.model.forward(self.t, self.dt_yr)
        if marks:
            marks[1].record()
        tm.ops.set_surface_enthalpy_from_temperature(self.surface_T())
        tm.step(self.dt_s)
        if marks:
            marks[2].record()
        self.t += self.dt_yr
        ls = getattr(tm.ops, "last_stats", None)
        return st, (int(ls.iterations) if ls is not None else None)

    def fields(self):
        """Level-0 u, v, H, the enthalpy (ny, nx, nz) and B, as NumPy arrays."""
        g = self.grid
        return {"u": g.state.u.data.cpu().numpy(), "v": g.state.v.data.cpu().numpy(),
                "H": g.state.H.data.cpu().numpy(), "E": self.thermal.enthalpy.cpu().numpy(),
                "B": g.rheology.B.data.cpu().numpy()}
