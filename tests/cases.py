"""Parity cases shared by the CPU and GPU tests: small grids that exercise every
solver, boundary, CPML kind and source kind, odd sizes and the medium split."""
from __future__ import annotations

import math

import numpy as np

from mpulse_b200 import abi, configs


def make_case(name: str, precision: int = abi.MP_FP64) -> abi.Config:
    spec = CASES[name]
    nx, ny, nz = spec.get("n", (20, 12, 28))
    # the medium Courant number: dt = 0.5 dx / c is unstable for the reference's
    # PLRC scheme with eps_inf = 1 and the 68.4 nm pole (test_stability.py)
    c = configs.base(nx, ny, nz, courant=configs.MEDIUM_COURANT)
    c.precision = precision
    c.solver = spec["solver"]
    c.boundary = spec.get("boundary", abi.MP_BOUNDARY_XY_PERIODIC)
    c.chi = spec.get("chi", 0.05)
    c.eps = spec.get("eps", 1.0)
    poles = spec.get("poles", configs.SILICA_POLES)
    for n in range(3):
        if n < len(poles):
            c.poles[n].eps, c.poles[n].delta, c.poles[n].om2 = poles[n]
        else:
            c.poles[n].eps, c.poles[n].delta, c.poles[n].om2 = 0.0, 0.0, 1.0
    c.medium_z0, c.medium_z1 = spec.get("medium", (0, nz + 1))
    c.eps_bg = spec.get("eps_bg", 1.0)
    c.cpml = spec.get("cpml", abi.MP_CPML_NONE)
    c.cpml_d = spec.get("cpml_d", 5)
    c.cpml_kappa_max = spec.get("kappa", 2.0)
    c.cpml_a_max = spec.get("amax", 0.1)
    c.cpml_sigma_max = spec.get("sigma", 40.0)
    srcs = spec.get("sources", ())
    c.n_sources = len(srcs)
    for q, kind in enumerate(srcs):
        s = c.sources[q]
        s.kind = kind
        s.distance = spec.get("src_d", 8)
        s.k[:] = (0.4, -0.3, 2 * math.pi / 0.8)
        s.H[:] = (0.2, 1.0, 0.0)
        s.H_bg[:] = (0.01, 0.0, 0.0)
        s.E_bg[:] = (0.0, 0.02, 0.0)
        s.ramp = 0.5
        s.width = 2.0
        s.offset = 6.0
        s.eps = 1.0
        s.length = 1.2
        s.waist = 0.2
        s.om0 = 2 * math.pi / 0.8
        s.t_shift = 0.5
        s.z_shift = -0.1
        s.phase = 0.1
        s.amp = 1.0
        for key, val in spec.get("src", {}).items():
            setattr(s, key, val)
    # the plasma plug-ins: "plasma" = (nu, mpa, Wion, K), "plasma_current" =
    # (em, gamma, rho_bg)
    if "plasma" in spec:
        c.plasma = 1
        c.plasma_nu, c.plasma_mpa, c.plasma_wion, c.plasma_k = spec["plasma"]
    if "plasma_current" in spec:
        c.plasma_current = 1
        c.plasma_em, c.plasma_gamma, c.plasma_rho_bg = spec["plasma_current"]
    return c


P = abi
CASES = {
    "plain_xy": dict(solver=P.MP_SOLVER_PLAIN),
    "plain_periodic": dict(solver=P.MP_SOLVER_PLAIN, boundary=P.MP_BOUNDARY_PERIODIC),
    "nl_periodic": dict(solver=P.MP_SOLVER_NL, boundary=P.MP_BOUNDARY_PERIODIC, chi=0.3, eps=1.5),
    "nl_xy": dict(solver=P.MP_SOLVER_NL, chi=0.3, eps=1.5),
    "lin_vacuum_cpmlz": dict(solver=P.MP_SOLVER_PLRC_LIN, poles=(), cpml=P.MP_CPML_Z),
    "lin_split_cpmlz_gauss": dict(solver=P.MP_SOLVER_PLRC_LIN, medium=(14, 40), cpml=P.MP_CPML_Z,
                                  sources=(P.MP_SOURCE_PLANE_GAUSS,)),
    "lin_all_wave_periodic": dict(solver=P.MP_SOLVER_PLRC_LIN, boundary=P.MP_BOUNDARY_PERIODIC,
                                  cpml=P.MP_CPML_ALL, cpml_d=4, sources=(P.MP_SOURCE_PLANE_WAVE,)),
    "nonlin_all_short": dict(solver=P.MP_SOLVER_PLRC_NONLIN, cpml=P.MP_CPML_ALL, cpml_d=4, chi=0.2,
                             medium=(10, 24), eps_bg=1.2, sources=(P.MP_SOURCE_SHORT_PULSE,)),
    "nonlin_three_poles": dict(solver=P.MP_SOLVER_PLRC_NONLIN, chi=0.2,
                               poles=configs.SILICA_POLES + (configs.lorentz_pole(0.3, 0.3, 0.01),),
                               eps=1.3, cpml=P.MP_CPML_Z, sources=(P.MP_SOURCE_PLANE_GAUSS,
                                                                   P.MP_SOURCE_PLANE_WAVE)),
    "nonlin_odd_sizes": dict(solver=P.MP_SOLVER_PLRC_NONLIN, n=(37, 13, 19), chi=0.1, cpml=P.MP_CPML_ALL,
                             cpml_d=3, medium=(5, 30), sources=(P.MP_SOURCE_PLANE_GAUSS,), src_d=6),
    "lin_thick_cpml_overlap": dict(solver=P.MP_SOLVER_PLRC_LIN, n=(9, 10, 11), cpml=P.MP_CPML_ALL, cpml_d=7),
    "nonlin_one_pole_periodic": dict(solver=P.MP_SOLVER_PLRC_NONLIN, boundary=P.MP_BOUNDARY_PERIODIC,
                                     poles=(configs.lorentz_pole(0.5, 0.1),), chi=0.4),
    # gauss_inject: Nt = 16 steps per spectral block for nz = 14.  The first
    # starts at t_off = 2 and is the only block (t_size 16): zero before, zero
    # after.  The second crosses two block boundaries and wraps in t.
    "lin_cpmlz_gauss_beam": dict(solver=P.MP_SOLVER_PLRC_LIN, n=(12, 10, 14), cpml=P.MP_CPML_Z, cpml_d=3,
                                 medium=(8, 40), sources=(P.MP_SOURCE_GAUSS_BEAM,), src_d=5,
                                 src=dict(t_size=16, t_off=2, length=0.15, width=0.08, k0=2 * math.pi / 0.8,
                                          time=0.1, shift=0.02, amp=0.7)),
    "nonlin_all_gauss_beam_blocks": dict(solver=P.MP_SOLVER_PLRC_NONLIN, n=(16, 8, 14), cpml=P.MP_CPML_ALL,
                                         cpml_d=3, chi=0.2, medium=(9, 40), sources=(P.MP_SOURCE_GAUSS_BEAM,),
                                         src_d=6, src=dict(t_size=40, t_off=0, length=0.2, width=0.1,
                                                           k0=2 * math.pi / 0.7, time=0.2, shift=-0.03,
                                                           amp=1.1, eps=1.2)),
    # x a multiple of 64: the B half runs its two-cell vector kernel; with
    # CPML on all faces its x-face (per cell), y-face (per row) and z-face
    # paths, and the injection plane, all run
    "vec_nonlin_all_short": dict(solver=P.MP_SOLVER_PLRC_NONLIN, n=(64, 12, 22), cpml=P.MP_CPML_ALL, cpml_d=4,
                                 chi=0.2, medium=(8, 40), eps_bg=1.2, sources=(P.MP_SOURCE_SHORT_PULSE,), src_d=6),
    "vec_lin_all_thick_wave": dict(solver=P.MP_SOLVER_PLRC_LIN, n=(128, 9, 13), cpml=P.MP_CPML_ALL, cpml_d=5,
                                   sources=(P.MP_SOURCE_PLANE_WAVE,), src_d=4),
    # x a multiple of 32 and y of 8: these run the TMA-staged kernels
    "tma_nonlin_all_short": dict(solver=P.MP_SOLVER_PLRC_NONLIN, n=(32, 16, 20), cpml=P.MP_CPML_ALL, cpml_d=4,
                                 chi=0.2, medium=(6, 30), sources=(P.MP_SOURCE_SHORT_PULSE,), src_d=5),
    "tma_lin_periodic_three_poles": dict(solver=P.MP_SOLVER_PLRC_LIN, n=(64, 8, 18),
                                         boundary=P.MP_BOUNDARY_PERIODIC, eps=1.3, cpml=P.MP_CPML_Z, cpml_d=3,
                                         poles=configs.SILICA_POLES + (configs.lorentz_pole(0.3, 0.3, 0.01),),
                                         sources=(P.MP_SOURCE_PLANE_WAVE,), src_d=5),
    "tma_plain_xy": dict(solver=P.MP_SOLVER_PLAIN, n=(32, 24, 12)),
    "tma_nl_xy": dict(solver=P.MP_SOLVER_NL, n=(64, 16, 10), chi=0.3, eps=1.5),
    "tma_lin_vacuum_cpmlz": dict(solver=P.MP_SOLVER_PLRC_LIN, n=(32, 8, 16), poles=(), cpml=P.MP_CPML_Z),
    # the plasma plug-ins: density (its conductivity in the E update) and
    # current, together with CPML, an injector, the medium split and Kerr;
    # the density alone; the current alone on a background density
    "plasma_nonlin_all_short": dict(solver=P.MP_SOLVER_PLRC_NONLIN, cpml=P.MP_CPML_ALL, cpml_d=4, chi=0.2,
                                    medium=(10, 24), eps_bg=1.2, sources=(P.MP_SOURCE_SHORT_PULSE,),
                                    plasma=(0.4, 3.0, 0.7, 2), plasma_current=(0.8, 0.3, 0.05)),
    "plasma_density_lin_periodic": dict(solver=P.MP_SOLVER_PLRC_LIN, boundary=P.MP_BOUNDARY_PERIODIC,
                                        plasma=(0.3, 5.0, 1.5, 3)),
    "plasma_current_lin_cpmlz": dict(solver=P.MP_SOLVER_PLRC_LIN, cpml=P.MP_CPML_Z, medium=(8, 40),
                                     sources=(P.MP_SOURCE_PLANE_GAUSS,), plasma_current=(1.3, 0.2, 0.4)),
    "vec_plasma_nonlin_all": dict(solver=P.MP_SOLVER_PLRC_NONLIN, n=(64, 6, 10), cpml=P.MP_CPML_ALL, cpml_d=2,
                                  chi=0.2, sources=(P.MP_SOURCE_PLANE_WAVE,), src_d=4,
                                  plasma=(0.4, 2.0, 0.9, 2), plasma_current=(0.9, 0.2, 0.1)),
}


def random_fields(cfg: abi.Config, seed: int, scale: float = 0.3, smooth: bool = False) -> dict:
    """Seeded initial fields in the plane layout.  `smooth` gives a sum of a
    few long-wavelength modes instead of grid-scale noise."""
    rng = np.random.default_rng(seed)
    shape = cfg.field_shape()
    out = {}
    for n in abi.FIELD_NAMES:
        if smooth:
            z, y, x = np.meshgrid(np.arange(shape[0]), np.arange(shape[1]), np.arange(shape[2]), indexing="ij")
            f = np.zeros(shape)
            for _ in range(3):
                kx = 2 * np.pi * rng.integers(0, 3) / shape[2]
                ky = 2 * np.pi * rng.integers(0, 3) / shape[1]
                kz = 2 * np.pi * rng.uniform(0.02, 0.1)
                f += rng.uniform(-1, 1) * np.cos(kx * x + ky * y + kz * z + rng.uniform(0, 6.28))
            out[n] = scale * f
        else:
            out[n] = scale * rng.standard_normal(shape)
    if cfg.boundary == abi.MP_BOUNDARY_PERIODIC:
        for n in out:  # ghost planes are images in a z-periodic grid
            out[n][0] = out[n][-2]
            out[n][-1] = out[n][1]
    return out


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
