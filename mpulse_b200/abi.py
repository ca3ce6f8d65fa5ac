"""ctypes mirror of include/mpulse_b200.h (mp_config and friends).

The layout here must match the C header field for field; a CPU test compares
``ctypes.sizeof`` and the defaults with the compiled library.
"""
from __future__ import annotations

import ctypes as C
import math

MP_ABI_VERSION = 2
MP_MAX_POLES = 3
MP_MAX_SOURCES = 4
MP_NOALLOC_MAX_PLANES = 16384

# mp_status
MP_OK = 0
MP_ERR_INVALID = -1
MP_ERR_CUDA = -2
MP_ERR_NO_MEMORY = -3
MP_ERR_NEWTON = -4
MP_ERR_NONFINITE = -5
MP_ERR_UNSUPPORTED = -6
MP_ERR_NAME = -7
MP_ERR_BOUNDS = -8

STATUS_NAMES = {
    MP_OK: "MP_OK",
    MP_ERR_INVALID: "MP_ERR_INVALID",
    MP_ERR_CUDA: "MP_ERR_CUDA",
    MP_ERR_NO_MEMORY: "MP_ERR_NO_MEMORY",
    MP_ERR_NEWTON: "MP_ERR_NEWTON",
    MP_ERR_NONFINITE: "MP_ERR_NONFINITE",
    MP_ERR_UNSUPPORTED: "MP_ERR_UNSUPPORTED",
    MP_ERR_NAME: "MP_ERR_NAME",
    MP_ERR_BOUNDS: "MP_ERR_BOUNDS",
}

MP_FP64, MP_FP32 = 0, 1
MP_SOLVER_PLAIN, MP_SOLVER_NL, MP_SOLVER_PLRC_LIN, MP_SOLVER_PLRC_NONLIN = 0, 1, 2, 3
MP_BOUNDARY_PERIODIC, MP_BOUNDARY_XY_PERIODIC = 0, 1
MP_CPML_NONE, MP_CPML_ALL, MP_CPML_Z = 0, 1, 2
MP_STAGING_AUTO, MP_STAGING_GLOBAL, MP_STAGING_TMA, MP_STAGING_FUSED = 0, 1, 2, 3
(MP_SOURCE_NONE, MP_SOURCE_PLANE_WAVE, MP_SOURCE_PLANE_GAUSS,
 MP_SOURCE_SHORT_PULSE, MP_SOURCE_FOCUSED_PULSE, MP_SOURCE_GAUSS_BEAM) = range(6)

MP_OBJ_E2_BOX, MP_OBJ_SZ_PLANE = 1, 2

FIELD_NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")
DESIGN_NAMES = ("DesignEps", "DesignDepsScale", "DesignChiScale")
PSI_NAMES = tuple(f"Psi{ri}{n}{c}" for ri in "RI" for n in (1, 2, 3) for c in "xyz")
PLASMA_NAMES = ("PlasmaDensity", "PlasmaJx", "PlasmaJy", "PlasmaJz")


class LorentzPole(C.Structure):
    _fields_ = [("eps", C.c_double), ("delta", C.c_double), ("om2", C.c_double)]


class Source(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("distance", C.c_int),
        ("k", C.c_double * 3),
        ("H", C.c_double * 3),
        ("H_bg", C.c_double * 3),
        ("E_bg", C.c_double * 3),
        ("ramp", C.c_double),
        ("width", C.c_double),
        ("offset", C.c_double),
        ("eps", C.c_double),
        ("length", C.c_double),
        ("waist", C.c_double),
        ("om0", C.c_double),
        ("t_shift", C.c_double),
        ("z_shift", C.c_double),
        ("phase", C.c_double),
        ("amp", C.c_double),
        ("t_size", C.c_int),
        ("t_off", C.c_int),
        ("k0", C.c_double),
        ("shift", C.c_double),
        ("time", C.c_double),
    ]


class Config(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int),
        ("nx", C.c_int),
        ("ny", C.c_int),
        ("nz", C.c_int),
        ("dx", C.c_double),
        ("dy", C.c_double),
        ("dz", C.c_double),
        ("dt", C.c_double),
        ("precision", C.c_int),
        ("solver", C.c_int),
        ("boundary", C.c_int),
        ("eps", C.c_double),
        ("chi", C.c_double),
        ("poles", LorentzPole * MP_MAX_POLES),
        ("medium_z0", C.c_int),
        ("medium_z1", C.c_int),
        ("eps_bg", C.c_double),
        ("cpml", C.c_int),
        ("cpml_d", C.c_int),
        ("cpml_kappa_max", C.c_double),
        ("cpml_a_max", C.c_double),
        ("cpml_sigma_max", C.c_double),
        ("n_sources", C.c_int),
        ("sources", Source * MP_MAX_SOURCES),
        ("newton_max_iter", C.c_int),
        ("newton_tol", C.c_double),
        ("staging", C.c_int),
        ("device", C.c_int),
        ("design_box", C.c_int * 6),
        ("plasma", C.c_int),
        ("plasma_nu", C.c_double),
        ("plasma_mpa", C.c_double),
        ("plasma_wion", C.c_double),
        ("plasma_k", C.c_int),
        ("plasma_current", C.c_int),
        ("plasma_em", C.c_double),
        ("plasma_gamma", C.c_double),
        ("plasma_rho_bg", C.c_double),
    ]

    def field_count(self) -> int:
        """Doubles in one host buffer of the plane layout: (nz+2) * ny * nx."""
        return (self.nz + 2) * self.ny * self.nx

    def field_shape(self):
        return (self.nz + 2, self.ny, self.nx)


class AdjointConfig(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("box", C.c_int * 6),
        ("steps", C.c_int),
        ("checkpoint_every", C.c_int),
        ("mem_budget", C.c_double),
    ]


MP_INIT_PULSE, MP_INIT_PLANE_GAUSS, MP_INIT_WAVE = 1, 2, 3


class Init(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("k", C.c_double * 3),
        ("B", C.c_double * 3),
        ("r0", C.c_double),
        ("z0", C.c_double),
        ("zc", C.c_double),
        ("C", C.c_double),
        ("eps", C.c_double),
        ("bound", C.c_int),
    ]


def default_init(kind: int) -> Init:
    """MakeParamMap defaults of pulse_init / gauss_init / wave_init
    (pulseinit.cpp:77-89, gaussinit.cpp:85-95, waveinit.cpp:63-74)."""
    q = Init()
    q.kind = kind
    q.k[:] = (1.0, 1.0, 1.0)
    q.B[:] = (1.0, 1.0, 1.0)
    q.r0 = q.z0 = q.zc = q.C = 1.0
    q.eps = 1.0
    q.bound = 0
    return q


def adjoint_config(kind: int, box, steps: int, checkpoint_every: int = 0, mem_budget: float = 0.0) -> AdjointConfig:
    a = AdjointConfig()
    a.kind = kind
    a.box[:] = tuple(box)
    a.steps = steps
    a.checkpoint_every = checkpoint_every
    a.mem_budget = mem_budget
    return a


def design_shape(c: Config):
    """(nz, ny, nx) extent of the design box, or None when it is empty."""
    b = c.design_box
    if b[0] > b[1]:
        return None
    return (b[5] - b[4] + 1, b[3] - b[2] + 1, b[1] - b[0] + 1)


def default_source(kind: int = MP_SOURCE_NONE) -> Source:
    """Parameter defaults of the injector plug-ins (incsource.cpp:84,
    sources.cpp:62-79 and :229-239, shortpulseinject.cpp:38-46)."""
    s = Source()
    s.kind = kind
    s.distance = 15
    s.k[:] = (0.0, 0.0, 1.0)
    s.H[:] = (0.0, 0.0, 0.0)
    s.ramp = 0.5
    s.width = 10.0
    s.offset = 40.0
    s.eps = 1.0
    s.length = 1.0
    s.waist = 1.0
    s.om0 = 2 * math.pi
    s.amp = 1.0
    s.t_size = 4096
    s.t_off = 0
    s.k0 = 2 * math.pi
    return s


def default_config() -> Config:
    """MPulse's ParameterValue defaults (globals.cpp:53-63 for dx/dt,
    fdtd_plrc.t:417-429, fdtd_plrc.cpp:463, cpml_border.cpp:146-149) on a 32^3
    grid; the same values as mp_config_defaults() in the C library."""
    c = Config()
    c.abi_version = MP_ABI_VERSION
    c.nx = c.ny = c.nz = 32
    c.dx = c.dy = c.dz = 0.1
    c.dt = 1e-2
    c.precision = MP_FP64
    c.solver = MP_SOLVER_PLRC_LIN
    c.boundary = MP_BOUNDARY_PERIODIC
    c.eps = 1.0
    c.chi = 0.1
    for n in range(MP_MAX_POLES):
        c.poles[n].eps = 0.0
        c.poles[n].delta = 0.0
        c.poles[n].om2 = 1.0
    c.medium_z0 = 0
    c.medium_z1 = 1 << 30
    c.eps_bg = 1.0
    c.cpml = MP_CPML_NONE
    c.cpml_d = 8
    c.cpml_kappa_max = 15.0
    c.cpml_a_max = 0.25
    c.cpml_sigma_max = 3.0
    c.n_sources = 0
    for n in range(MP_MAX_SOURCES):
        c.sources[n] = default_source()
    c.newton_max_iter = 64
    c.newton_tol = 1e-9
    c.staging = MP_STAGING_AUTO
    c.device = 0
    c.design_box[:] = (1, 0, 1, 0, 1, 0)
    c.plasma = 0
    c.plasma_nu = c.plasma_mpa = c.plasma_wion = 1.0
    c.plasma_k = 5
    c.plasma_current = 0
    c.plasma_em = 1.0
    c.plasma_gamma = 0.1
    c.plasma_rho_bg = 0.0
    return c


def config_to_dict(c: Config) -> dict:
    """Plain-dict view of a Config (for logs and fixtures)."""
    def conv(v):
        if isinstance(v, C.Structure):
            return {f: conv(getattr(v, f)) for f, _ in v._fields_}
        if isinstance(v, C.Array):
            return [conv(x) for x in v]
        return v
    return conv(c)


def config_from_dict(d: dict) -> Config:
    c = default_config()

    def fill(obj, dd):
        for f, _ in obj._fields_:
            if f not in dd:
                continue
            v = getattr(obj, f)
            if isinstance(v, C.Structure):
                fill(v, dd[f])
            elif isinstance(v, C.Array):
                for n, x in enumerate(dd[f]):
                    if isinstance(v[n], C.Structure):
                        fill(v[n], x)
                    else:
                        v[n] = x
            else:
                setattr(obj, f, dd[f])
    fill(c, d)
    return c
