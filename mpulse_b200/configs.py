"""The five workloads this path is measured and checked on, as mp_configs, plus
the host-side initial fields they need.

Units are MPulse's normalised ones: c = eps0 = mu0 = 1 with lengths in um, so
a time of 1 is 1 um / c = 3.336 fs.  A Lorentz pole of strength de at
resonance wavelength lam with damping gamma = 1e-3 * omega_res maps onto MPulse's
parameters (fdtd_plrc.t:419-429, fdtd_plrc.h:85-90) as
    L<n>eps = de,  L<n>Om2 = (2 pi / lam)^2,  L<n>delta = gamma / 2.
A pole slot that must exist but carry no medium gets eps = 0, om2 = 1
(MPulse rejects om2 = 0, fdtd_plrc.t:20-24).
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

C_UM_PER_FS = 0.299792458  # c in um / fs


def fs_to_time(fs: float) -> float:
    return fs * C_UM_PER_FS


def lorentz_pole(de: float, lam_um: float, damping: float = 1e-3):
    om = 2 * math.pi / lam_um
    return (de, 0.5 * damping * om, om * om)  # (eps, delta, om2)


# fused-silica-like two-pole medium of the workloads
SILICA_POLES = (lorentz_pole(0.6961663, 0.0684), lorentz_pole(0.4079426, 0.1162))

# Courant number of the workloads with the two-pole medium.  MPulse's PLRC
# update (fdtd_plrc.cpp:94-261) with eps_inf = 1 and the 68.4 nm pole, whose
# resonance turns by omega dt = 1.84 rad per step at dx = 40 nm, amplifies
# grid-scale perturbations at dt = 0.5 dx / c (about x1e4 per 25 steps, in the
# reference and in this implementation alike) and is stable at 0.45; the
# workloads with that medium therefore run at dt = 0.45 dx / c.
MEDIUM_COURANT = 0.45


def sigma_max_for(R: float, d: int, dx: float, m: int = 3) -> float:
    """Polynomial-graded PML conductivity for a normal-incidence reflection R:
    sigma_max = -(m + 1) ln R / (2 d dx)."""
    return -(m + 1) * math.log(R) / (2 * d * dx)


def field_fwhm_to_t0(fwhm_fs: float) -> float:
    """Intensity FWHM (fs) -> 1/e half-width t0 of the field envelope
    exp(-(t / t0)^2), in normalised time."""
    return fs_to_time(fwhm_fs) / math.sqrt(2 * math.log(2))


def _set_poles(c: abi.Config, poles):
    for n in range(abi.MP_MAX_POLES):
        if n < len(poles):
            c.poles[n].eps, c.poles[n].delta, c.poles[n].om2 = poles[n]
        else:
            c.poles[n].eps, c.poles[n].delta, c.poles[n].om2 = 0.0, 0.0, 1.0


def base(nx, ny, nz, dx=0.04, courant=0.5) -> abi.Config:
    c = abi.default_config()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dx = c.dy = c.dz = dx
    c.dt = courant * dx
    return c


def c1_vacuum_pulse(precision=abi.MP_FP64, n=64) -> abi.Config:
    """Plain vacuum Yee, 64^3, dx = 40 nm, dt = 0.5 dx / c, periodic x/y,
    8-cell CPML on the z faces (cubic grading, sigma_max for R = 1e-6).
    MPulse's fdtd-plain cannot host CPML (fieldsolver.h:198-216), so this is
    fdtd-plrc-lin with no active pole, which updates vacuum cells with the same
    arithmetic."""
    c = base(n, n, n)
    c.precision = precision
    c.solver = abi.MP_SOLVER_PLRC_LIN
    c.boundary = abi.MP_BOUNDARY_XY_PERIODIC
    _set_poles(c, ())
    c.cpml = abi.MP_CPML_Z
    c.cpml_d = 8
    c.cpml_kappa_max = 1.0
    c.cpml_a_max = 0.0
    c.cpml_sigma_max = sigma_max_for(1e-6, 8, c.dz)
    return c


def c2_linear_plrc(precision=abi.MP_FP32, n=128, medium_z0=40, src_d=16) -> abi.Config:
    """Linear dispersive PLRC, 128^3 (dt = MEDIUM_COURANT dx / c): vacuum for z < 40, two-pole Lorentz medium
    for z >= 40, 10-cell CPML on the z faces, Ex plane-wave pulse (lambda0 =
    800 nm, 10 fs FWHM) injected at z = 16 by plane_gauss_inject."""
    c = base(n, n, n, courant=MEDIUM_COURANT)
    c.precision = precision
    c.solver = abi.MP_SOLVER_PLRC_LIN
    c.boundary = abi.MP_BOUNDARY_XY_PERIODIC
    _set_poles(c, SILICA_POLES)
    c.eps = 1.0
    c.medium_z0, c.medium_z1 = medium_z0, n + 1
    c.cpml = abi.MP_CPML_Z
    c.cpml_d = 10
    c.cpml_kappa_max = 1.0
    c.cpml_a_max = 0.0
    c.cpml_sigma_max = sigma_max_for(1e-6, 10, c.dz)
    k0 = 2 * math.pi / 0.8
    width = k0 * field_fwhm_to_t0(10.0)      # envelope width in phase units
    c.n_sources = 1
    s = c.sources[0]
    s.kind = abi.MP_SOURCE_PLANE_GAUSS
    s.distance = src_d
    s.k[:] = (0.0, 0.0, k0)
    s.H[:] = (0.0, 1.0, 0.0)
    s.width = width
    s.offset = 3.0 * width
    s.eps = 1.0
    return c


def c3_plrc_kerr(precision=abi.MP_FP32, nx=256, ny=256, nz=512, medium_z0=64, focus_z=200, src_d=20,
                 chi=0.01) -> abi.Config:
    """PLRC + Kerr, 256 x 256 x 512 (dt = MEDIUM_COURANT dx / c), 12-cell CPML on all six faces, two-pole
    medium with chi3 E0^2 = 0.01 filling z >= 64, focused Gaussian pulse
    (waist 2 um at z = 200, lambda0 = 800 nm, 20 fs FWHM, peak E0 = 1) from the
    paraxial short-pulse closed form (shortpulseinject)."""
    c = base(nx, ny, nz, courant=MEDIUM_COURANT)
    c.precision = precision
    c.solver = abi.MP_SOLVER_PLRC_NONLIN
    c.boundary = abi.MP_BOUNDARY_XY_PERIODIC
    _set_poles(c, SILICA_POLES)
    c.eps = 1.0
    c.chi = chi
    c.medium_z0, c.medium_z1 = medium_z0, nz + 1
    c.cpml = abi.MP_CPML_ALL
    c.cpml_d = 12
    c.cpml_kappa_max = 1.0
    c.cpml_a_max = 0.0
    c.cpml_sigma_max = sigma_max_for(1e-6, 12, c.dz)
    c.n_sources = 1
    s = c.sources[0]
    s.kind = abi.MP_SOURCE_SHORT_PULSE
    s.distance = src_d
    s.length = field_fwhm_to_t0(20.0)
    s.waist = 2.0
    s.om0 = 2 * math.pi / 0.8
    centre_z = 0.5 * (nz + 1)
    s.z_shift = (focus_z - centre_z) * c.dz
    z_inj = (src_d - centre_z) * c.dz - s.z_shift
    s.t_shift = 3.0 * s.length - z_inj
    s.amp = 1.0
    s.eps = 1.0
    return c


def pulse_init_fields(cfg: abi.Config, k: float, z0: float, zc: float, r0: float = 1e6, C: float = 0.0,
                      bx: float = 0.0, by: float = 1.0, bound: int = 0) -> dict:
    """Initial fields of GaussPulseInit::init (pulseinit.cpp:7-74) in the plane
    layout: a Gaussian beam pulse with Ex = by*amp_e, Ey = -bx*amp_e,
    Bx = bx*amp_b, By = by*amp_b, staggered by half a cell in z for B.
    MPulse writes ghost cells too; here x/y are periodic and only the z ghost
    planes are stored."""
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    dx, dy, dz = cfg.dx, cfg.dy, cfg.dz
    ex_amp, ey_amp = by, -bx
    xh = 0.5 * (nx + 1)
    yh = 0.5 * (ny + 1)
    i = np.arange(1, nx + 1, dtype=np.float64)
    j = np.arange(1, ny + 1, dtype=np.float64)
    kk = np.arange(0, nz + 2, dtype=np.float64)
    ii, jj = np.meshgrid(i, j)  # (ny, nx)
    rre = ((ii - xh) ** 2 * dx * dx + (jj - yh) ** 2 * dy * dy) / (r0 * r0)
    rrb = ((ii + 0.5 - xh) ** 2 * dx * dx + (jj + 0.5 - yh) ** 2 * dy * dy) / (r0 * r0)
    nze = kk * dz - zc
    nzb = (kk + 0.5) * dz - zc
    kze = kk * (dz * k)
    kzb = (kk + 0.5) * (dz * k)
    ampe = np.cos(kze[:, None, None] - C * rre[None]) * np.exp(-nze[:, None, None] ** 2 / (z0 * z0) - rre[None])
    ampb = np.cos(kzb[:, None, None] - C * rrb[None]) * np.exp(-nzb[:, None, None] ** 2 / (z0 * z0) - rrb[None])
    kmask = np.zeros(nz + 2, dtype=bool)
    kmask[bound:nz + 2 - bound] = True
    m = kmask[:, None, None]
    out = {
        "Ex": np.where(m, ex_amp * ampe, 0.0), "Ey": np.where(m, ey_amp * ampe, 0.0),
        "Ez": np.zeros_like(ampe),
        "Bx": np.where(m, bx * ampb, 0.0), "By": np.where(m, by * ampb, 0.0), "Bz": np.zeros_like(ampb),
    }
    return {n: np.ascontiguousarray(v) for n, v in out.items()}


def c1_initial_fields(cfg: abi.Config) -> dict:
    """The Ex-polarised plane-wave pulse of the vacuum workload: lambda0 =
    800 nm, 5 fs intensity FWHM, centred at z = 20 cells (pulse_init with
    r0 -> infinity)."""
    k0 = 2 * math.pi / 0.8
    z0 = field_fwhm_to_t0(5.0)  # spatial 1/e half-width = c t0
    return pulse_init_fields(cfg, k=k0, z0=z0, zc=20 * cfg.dz)


def c4_adjoint(precision=abi.MP_FP64, n=96, seed=0) -> tuple:
    """Adjoint-gradient workload, 96^3 (dt = MEDIUM_COURANT dx / c), 10-cell
    CPML on all faces, linear single-pole Lorentz medium (Delta eps = 0.5,
    lambda_res = 100 nm, gamma = 1e-3 omega_res) everywhere, a 32^3 design
    region at the centre whose eps_inf is drawn i.i.d. uniform in [1, 4] from
    torch.Generator().manual_seed(seed), an Ex plane-wave pulse (lambda0 =
    800 nm, 10 fs FWHM) injected at z = 14, and the objective
    J = sum_t sum |E|^2 dt over the 8^3 monitor box centred at (48, 48, 80),
    1500 steps with a checkpoint every 50.
    Returns (config, {design map name: array}, adjoint config)."""
    import torch

    c = base(n, n, n, courant=MEDIUM_COURANT)
    c.precision = precision
    c.solver = abi.MP_SOLVER_PLRC_LIN
    c.boundary = abi.MP_BOUNDARY_XY_PERIODIC
    _set_poles(c, (lorentz_pole(0.5, 0.1),))
    c.eps = 1.0
    c.medium_z0, c.medium_z1 = 0, n + 1
    c.cpml = abi.MP_CPML_ALL
    c.cpml_d = 10
    c.cpml_kappa_max = 1.0
    c.cpml_a_max = 0.0
    c.cpml_sigma_max = sigma_max_for(1e-6, 10, c.dz)
    k0 = 2 * math.pi / 0.8
    width = k0 * field_fwhm_to_t0(10.0)
    c.n_sources = 1
    s = c.sources[0]
    s.kind = abi.MP_SOURCE_PLANE_GAUSS
    s.distance = 14
    s.k[:] = (0.0, 0.0, k0)
    s.H[:] = (0.0, 1.0, 0.0)
    s.width = width
    s.offset = 3.0 * width
    s.eps = 1.0
    lo, hi = n // 2 - 15, n // 2 + 16          # 32 cells centred on n/2 + 1/2
    c.design_box[:] = (lo, hi, lo, hi, lo, hi)
    g = torch.Generator().manual_seed(seed)
    eps = 1.0 + 3.0 * torch.rand((32, 32, 32), generator=g, dtype=torch.float64)
    m = n // 2
    adj = abi.adjoint_config(abi.MP_OBJ_E2_BOX, (m - 3, m + 4, m - 3, m + 4, 77, 84), 1500, checkpoint_every=50)
    return c, {"DesignEps": eps.numpy()}, adj


def c5_adjoint(precision=abi.MP_FP32, nx=512, ny=512, nz=768, steps=6000, seed=0, design=(128, 128, 64),
               design_z0=320, sz_plane=700, src_d=20, cpml_d=16, medium_z0=64) -> tuple:
    """Large nonlinear adjoint workload, 512 x 512 x 768 (dt = MEDIUM_COURANT
    dx / c), 16-cell CPML on all faces, two-pole Lorentz medium with Kerr
    chi3 E0^2 = 0.02 filling z >= 64, a design region of 128 x 128 x 64 cells
    centred in x / y from z = 320 with eps_inf uniform in [1, 4] and a chi
    factor uniform in [0.5, 1.5] (torch.Generator().manual_seed(seed)), a
    focused pulse (waist 3 um at the design region's centre, lambda0 = 800 nm,
    20 fs FWHM, the short-pulse closed form) injected at z = 20, and the
    objective J = sum_t Sz dt dA through the plane z = 700; checkpoints within
    a 120 GB budget.  Returns (config, {design map name: array}, adjoint config)."""
    import torch

    c = c3_plrc_kerr(precision, nx=nx, ny=ny, nz=nz, medium_z0=medium_z0, focus_z=design_z0 + design[2] // 2,
                     src_d=src_d, chi=0.02)
    c.cpml_d = cpml_d
    c.cpml_sigma_max = sigma_max_for(1e-6, cpml_d, c.dz)
    c.sources[0].waist = 3.0
    bx, by, bz = design
    x0, y0 = nx // 2 - bx // 2 + 1, ny // 2 - by // 2 + 1
    c.design_box[:] = (x0, x0 + bx - 1, y0, y0 + by - 1, design_z0, design_z0 + bz - 1)
    g = torch.Generator().manual_seed(seed)
    eps = 1.0 + 3.0 * torch.rand((bz, by, bx), generator=g, dtype=torch.float64)
    chi = 0.5 + torch.rand((bz, by, bx), generator=g, dtype=torch.float64)
    adj = abi.adjoint_config(abi.MP_OBJ_SZ_PLANE, (1, nx, 1, ny, sz_plane, sz_plane), steps, mem_budget=120e9)
    return c, {"DesignEps": eps.numpy(), "DesignChiScale": chi.numpy()}, adj
