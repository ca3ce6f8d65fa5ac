"""TEST INFRASTRUCTURE ONLY: ctypes binding of the C oracle (liboracle.so) and
helpers that run the reference build (_ref/mpulse_ref) on an mp_config.

Imported by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline
leg, and nowhere else.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile

import numpy as np

from mpulse_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "mpulse_ref")
REF_BIN_FAST = os.path.join(HERE, "_ref", "mpulse_ref_fast")
REF_BIN_GPU = os.path.join(HERE, "_ref", "mpulse_ref_gpu")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle not built: run `make -C {HERE}`")
        L = C.CDLL(LIB_PATH)
        L.mpo_create.argtypes = [C.POINTER(abi.Config), C.POINTER(C.c_void_p)]
        L.mpo_create.restype = C.c_int
        L.mpo_destroy.argtypes = [C.c_void_p]
        L.mpo_destroy.restype = None
        L.mpo_create_error.restype = C.c_char_p
        for f in (L.mpo_upload, L.mpo_download):
            f.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.c_size_t]
            f.restype = C.c_int
        L.mpo_step.argtypes = [C.c_void_p, C.c_int]
        L.mpo_step.restype = C.c_int
        L.mpo_get_time.argtypes = [C.c_void_p]
        L.mpo_get_time.restype = C.c_longlong
        L.mpo_set_time.argtypes = [C.c_void_p, C.c_longlong]
        L.mpo_set_time.restype = None
        L.mpo_faddeeva.argtypes = [C.POINTER(C.c_double)] * 4 + [C.c_size_t]
        L.mpo_faddeeva.restype = None
        L.mpo_short_pulse.argtypes = [C.c_double] * 9 + [C.POINTER(C.c_double)]
        L.mpo_short_pulse.restype = None
        L.mpo_source_field.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_longlong, C.POINTER(C.c_double)]
        L.mpo_source_field.restype = C.c_int
        L.mpo_field_energy.argtypes = [C.c_void_p]
        L.mpo_field_energy.restype = C.c_double
        L.mpo_objective.argtypes = [C.c_void_p, C.POINTER(abi.AdjointConfig), C.POINTER(C.c_double)]
        L.mpo_objective.restype = C.c_int
        L.mpo_kappa.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_size_t]
        L.mpo_kappa.restype = C.c_int
        L.mpo_cpml_count.argtypes = [C.c_void_p, C.c_int]
        L.mpo_cpml_count.restype = C.c_int
        L.mpo_cpml_layer.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.c_size_t, C.POINTER(C.c_double)]
        L.mpo_cpml_layer.restype = C.c_int
        L.mpo_plrc_coefficients.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.mpo_plrc_coefficients.restype = None
        L.mpo_initialize.argtypes = [C.c_void_p, C.POINTER(abi.Init)]
        L.mpo_initialize.restype = C.c_int
        L.mpo_follow_max.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_double)]
        L.mpo_follow_max.restype = C.c_int
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleSim:
    """FP64 CPU restatement of the MPulse step for one mp_config."""

    def __init__(self, cfg: abi.Config):
        self.cfg = cfg
        self.h = None
        h = C.c_void_p()
        rc = lib().mpo_create(C.byref(cfg), C.byref(h))
        if rc != abi.MP_OK:
            raise ValueError(f"mpo_create: {abi.STATUS_NAMES.get(rc, rc)}: "
                             f"{lib().mpo_create_error().decode()}")
        self.h = h

    def close(self):
        if self.h:
            lib().mpo_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        rc = lib().mpo_upload(self.h, name.encode(), _dptr(a), a.size)
        if rc != abi.MP_OK:
            raise ValueError(f"mpo_upload({name}): {rc}")

    def download(self, name: str) -> np.ndarray:
        out = np.empty(self.cfg.field_count(), dtype=np.float64)
        rc = lib().mpo_download(self.h, name.encode(), _dptr(out), out.size)
        if rc != abi.MP_OK:
            raise ValueError(f"mpo_download({name}): {rc}")
        return out.reshape(self.cfg.field_shape())

    def step(self, n: int = 1) -> int:
        return lib().mpo_step(self.h, n)

    @property
    def time(self) -> int:
        return lib().mpo_get_time(self.h)

    @time.setter
    def time(self, t: int):
        lib().mpo_set_time(self.h, t)

    def field_energy(self) -> float:
        return lib().mpo_field_energy(self.h)

    def upload_design(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        rc = lib().mpo_upload(self.h, name.encode(), _dptr(a), a.size)
        if rc != abi.MP_OK:
            raise ValueError(f"mpo_upload({name}): {rc}")

    def objective(self, adj: abi.AdjointConfig) -> float:
        """Runs adj.steps steps and returns J (mp_objective's definition)."""
        J = C.c_double()
        rc = lib().mpo_objective(self.h, C.byref(adj), C.byref(J))
        if rc != abi.MP_OK:
            raise ValueError(f"mpo_objective: {abi.STATUS_NAMES.get(rc, rc)}")
        return J.value

    def kappa(self, isH: int, dim: int) -> np.ndarray:
        n = (self.cfg.nx, self.cfg.ny, self.cfg.nz)[dim] + 2
        out = np.empty(n)
        assert lib().mpo_kappa(self.h, isH, dim, _dptr(out), n) == abi.MP_OK
        return out

    def cpml_layers(self, isH: int):
        """[(dir, dim, lo[3], hi[3], b, c, delta)] of the CPML currents."""
        out = []
        for l in range(lib().mpo_cpml_count(self.h, isH)):
            info = (C.c_int * 8)()
            d = C.c_double()
            dummy = np.empty(1)
            lib().mpo_cpml_layer(self.h, isH, l, info, _dptr(dummy), _dptr(dummy), 0, C.byref(d))
            length = info[5 + info[1]] - info[2 + info[1]] + 1
            b = np.empty(length)
            c = np.empty(length)
            assert lib().mpo_cpml_layer(self.h, isH, l, info, _dptr(b), _dptr(c), length, C.byref(d)) == abi.MP_OK
            out.append((info[0], info[1], tuple(info[2:5]), tuple(info[5:8]), b, c, d.value))
        return out

    def plrc_coefficients(self) -> dict:
        o = np.empty(20)
        lib().mpo_plrc_coefficients(self.h, _dptr(o))
        z = lambda a: o[a:a + 6:2] + 1j * o[a + 1:a + 6:2]  # noqa: E731
        return {"dchi0": z(0), "dxi0": z(6), "crec": z(12), "sumChi0": o[18], "sumXi0": o[19]}

    def initialize(self, init: abi.Init):
        rc = lib().mpo_initialize(self.h, C.byref(init))
        if rc != abi.MP_OK:
            raise ValueError(f"mpo_initialize: {rc}")

    def follow_max(self, field: str, dim: int, pos, ipos: int):
        p = (C.c_int * 3)(*pos)
        ip = C.c_int(ipos)
        out = C.c_double()
        rc = lib().mpo_follow_max(self.h, field.encode(), dim, p, C.byref(ip), C.byref(out))
        if rc != abi.MP_OK:
            raise ValueError(f"mpo_follow_max: {rc}")
        return ip.value, out.value

    def source_field(self, src: int, which: int, i: int, j: int, l: int, time: int):
        out = np.zeros(3)
        rc = lib().mpo_source_field(self.h, src, which, i, j, l, time, _dptr(out))
        if rc != abi.MP_OK:
            raise ValueError("mpo_source_field")
        return out


def short_pulse(length, width, om0, phase, eps, x, y, z, t) -> np.ndarray:
    """Re and Im of Efunc, Bfunc(bx) and Bfunc(by) of the short-pulse closed
    form at one point (mpo_short_pulse)."""
    out = (C.c_double * 6)()
    lib().mpo_short_pulse(length, width, om0, phase, eps, x, y, z, t, out)
    return np.array(out[:])


def faddeeva(z: np.ndarray) -> np.ndarray:
    z = np.asarray(z, dtype=np.complex128).reshape(-1)
    re = np.ascontiguousarray(z.real)
    im = np.ascontiguousarray(z.imag)
    wr = np.empty_like(re)
    wi = np.empty_like(im)
    lib().mpo_faddeeva(_dptr(re), _dptr(im), _dptr(wr), _dptr(wi), z.size)
    return wr + 1j * wi


# --------------------------------------------------------------------------
# The reference build: setup-file writer and runner.

_SOLVER_NAMES = {
    abi.MP_SOLVER_PLAIN: "fdtd-plain",
    abi.MP_SOLVER_NL: "fdtd-nl",
    abi.MP_SOLVER_PLRC_LIN: "fdtd-plrc-masked-lin",
    abi.MP_SOLVER_PLRC_NONLIN: "fdtd-plrc-masked-nonlin",
}


def _fmt(x) -> str:
    return repr(float(x))


def init_block(init: abi.Init) -> str:
    """The setup-file block of a field initialiser (fieldsim.cpp:157-168)."""
    if init.kind == abi.MP_INIT_PULSE:
        return (f"pulse_init {{ k {_fmt(init.k[2])} r0 {_fmt(init.r0)} z0 {_fmt(init.z0)} zc {_fmt(init.zc)} "
                f"C {_fmt(init.C)} Bx {_fmt(init.B[0])} By {_fmt(init.B[1])} bound {init.bound} }}")
    ks = f"kx {int(init.k[0])} ky {int(init.k[1])} kz {int(init.k[2])}"
    bs = f"Bx {_fmt(init.B[0])} By {_fmt(init.B[1])} Bz {_fmt(init.B[2])}"
    if init.kind == abi.MP_INIT_PLANE_GAUSS:
        return f"gauss_init {{ {ks} {bs} }}"
    return f"wave_init {{ {ks} {bs} eps {_fmt(init.eps)} }}"


def setup_text(cfg: abi.Config, steps: int, init_file: str | None = None, solver_name: str | None = None,
               extra: str = "", inits: str = "", boundary: str | None = None) -> str:
    """MPulse setup file (rebuild.cpp grammar) describing `cfg`.  `solver_name`
    replaces the solver block's name (e.g. "fdtd-gpu-plrc-nonlin" for the B200
    plug-in, which reads the same keys); `extra` is appended to its body;
    `boundary` replaces the boundary block (e.g. the harness's
    "slab_xy_periodic { z0 .. z1 .. }")."""
    g = (f"globals {{ grid-x {cfg.nx} grid-y {cfg.ny} grid-z {cfg.nz} "
         f"grid-dx {_fmt(cfg.dx)} grid-dy {_fmt(cfg.dy)} grid-dz {_fmt(cfg.dz)} "
         f"dt {_fmt(cfg.dt)} T-total {steps} }}\n")
    bnd = boundary or ("single_periodic { }" if cfg.boundary == abi.MP_BOUNDARY_PERIODIC
                       else "single_xy_periodic { }")
    solver = solver_name or _SOLVER_NAMES[cfg.solver]
    body = [f"eps {_fmt(cfg.eps)}"]
    if cfg.solver in (abi.MP_SOLVER_NL, abi.MP_SOLVER_PLRC_NONLIN):
        body.append(f"chi {_fmt(cfg.chi)}")
    if cfg.solver in (abi.MP_SOLVER_PLRC_LIN, abi.MP_SOLVER_PLRC_NONLIN):
        for n in range(3):
            p = cfg.poles[n]
            body.append(f"L{n+1}eps {_fmt(p.eps)} L{n+1}delta {_fmt(p.delta)} L{n+1}Om2 {_fmt(p.om2)}")
        body.append(f"medium_z0 {cfg.medium_z0} medium_z1 {cfg.medium_z1} eps_bg {_fmt(cfg.eps_bg)}")
        if cfg.cpml != abi.MP_CPML_NONE:
            name = "cpml_border" if cfg.cpml == abi.MP_CPML_ALL else "cpml_border_1d"
            body.append(f"{name} {{ d {cfg.cpml_d} kappaMax {_fmt(cfg.cpml_kappa_max)} "
                        f"aMax {_fmt(cfg.cpml_a_max)} sigmaMax {_fmt(cfg.cpml_sigma_max)} }}")
        for n in range(cfg.n_sources):
            s = cfg.sources[n]
            if s.kind in (abi.MP_SOURCE_PLANE_WAVE, abi.MP_SOURCE_PLANE_GAUSS):
                kw = [f"d {s.distance}", f"kx {_fmt(s.k[0])} ky {_fmt(s.k[1])} kz {_fmt(s.k[2])}",
                      f"Hx {_fmt(s.H[0])} Hy {_fmt(s.H[1])} Hz {_fmt(s.H[2])}", f"eps {_fmt(s.eps)}"]
                if s.kind == abi.MP_SOURCE_PLANE_WAVE:
                    kw.append(f"Hx_bg {_fmt(s.H_bg[0])} Hy_bg {_fmt(s.H_bg[1])} Hz_bg {_fmt(s.H_bg[2])}")
                    kw.append(f"Ex_bg {_fmt(s.E_bg[0])} Ey_bg {_fmt(s.E_bg[1])} Ez_bg {_fmt(s.E_bg[2])}")
                    kw.append(f"ramp {_fmt(s.ramp)}")
                    body.append("wave_inject { " + " ".join(kw) + " }")
                else:
                    kw.append(f"width {_fmt(s.width)} offset {_fmt(s.offset)}")
                    body.append("plane_gauss_inject { " + " ".join(kw) + " }")
            elif s.kind == abi.MP_SOURCE_SHORT_PULSE:
                body.append("short_pulse_inject { " + " ".join([
                    f"d {s.distance}", f"length {_fmt(s.length)}", f"width {_fmt(s.waist)}",
                    f"om0 {_fmt(s.om0)}", f"TShift {_fmt(s.t_shift)}", f"ZShift {_fmt(s.z_shift)}",
                    f"Phase {_fmt(s.phase)}", f"amp {_fmt(s.amp)}", f"eps {_fmt(s.eps)}"]) + " }")
            elif s.kind == abi.MP_SOURCE_GAUSS_BEAM:
                body.append("gauss_inject { " + " ".join([
                    f"d {s.distance}", f"SizeT {s.t_size}", f"length {_fmt(s.length)}",
                    f"width {_fmt(s.width)}", f"k0 {_fmt(s.k0)}", f"Shift {_fmt(s.shift)}",
                    f"Time {_fmt(s.time)}", f"amp {_fmt(s.amp)}", f"eps {_fmt(s.eps)}",
                    f"toff {s.t_off}"]) + " }")
            else:
                raise ValueError(f"source kind {s.kind} has no runnable reference plug-in")
        # the plasma plug-ins (fdtd_plrc.t:431-436): the density is an E-side
        # optional field, the current is listed after the other currents
        if cfg.plasma:
            body.append(f"plasma {{ nu {_fmt(cfg.plasma_nu)} mpa {_fmt(cfg.plasma_mpa)} "
                        f"Wion {_fmt(cfg.plasma_wion)} K {cfg.plasma_k} }}")
        if cfg.plasma_current:
            body.append(f"plasma_current {{ em {_fmt(cfg.plasma_em)} gamma {_fmt(cfg.plasma_gamma)} "
                        f"rho_bg {_fmt(cfg.plasma_rho_bg)} }}")
    if extra:
        body.append(extra)
    init = f"raw_init {{ file {init_file} }}\n" if init_file else ""
    if inits:
        init += "  " + inits + "\n"
    return g + "fieldsim {\n  " + bnd + "\n  " + solver + " { " + " ".join(body) + " }\n  " + init + "}\n"


def plane_to_full(cfg: abi.Config, plane: np.ndarray) -> np.ndarray:
    """Plane layout -> MPulse's (nx+2, ny+2, nz+2) C-order grid, x/y ghosts
    filled with the periodic images."""
    p = np.asarray(plane).reshape(cfg.field_shape())
    full = np.zeros((cfg.nx + 2, cfg.ny + 2, cfg.nz + 2))
    inner = p.transpose(2, 1, 0)  # (nx, ny, nz+2)
    full[1:-1, 1:-1, :] = inner
    full[0, :, :] = full[-2, :, :]
    full[-1, :, :] = full[1, :, :]
    full[:, 0, :] = full[:, -2, :]
    full[:, -1, :] = full[:, 1, :]
    if cfg.boundary == abi.MP_BOUNDARY_PERIODIC:
        full[:, :, 0] = full[:, :, -2]
        full[:, :, -1] = full[:, :, 1]
    return full


def full_to_plane(cfg: abi.Config, full: np.ndarray) -> np.ndarray:
    f = np.asarray(full).reshape(cfg.nx + 2, cfg.ny + 2, cfg.nz + 2)
    return np.ascontiguousarray(f[1:-1, 1:-1, :].transpose(2, 1, 0))


def run_reference(cfg: abi.Config, steps: int, init_fields: dict | None = None,
                  names=abi.FIELD_NAMES, binary: str = REF_BIN, workdir: str | None = None,
                  solver_name: str | None = None, extra: str = "", inits: str = "", boundary: str | None = None):
    """Runs the reference build for `steps` steps from the given initial fields
    (plane layout; missing components are zero) and returns
    ({name: plane-layout array}, timing dict).  With binary=REF_BIN_GPU and a
    "fdtd-gpu-*" solver_name, MPulse's own driver runs the B200 plug-in."""
    if not os.path.exists(binary):
        raise RuntimeError(f"reference build missing: run `make -C {HERE} ref gpuref`")
    tmp = workdir or tempfile.mkdtemp(prefix="mpref_")
    init_path = None
    if init_fields:
        init_path = os.path.join(tmp, "init.bin")
        with open(init_path, "wb") as f:
            for n in abi.FIELD_NAMES:
                plane = init_fields.get(n)
                full = (plane_to_full(cfg, plane) if plane is not None
                        else np.zeros((cfg.nx + 2, cfg.ny + 2, cfg.nz + 2)))
                f.write(np.ascontiguousarray(full).tobytes())
    setup = os.path.join(tmp, "setup.dat")
    with open(setup, "w") as f:
        f.write(setup_text(cfg, steps, init_path, solver_name=solver_name, extra=extra, inits=inits,
                           boundary=boundary))
    r = subprocess.run([binary, setup, tmp, *names], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed ({r.returncode}): {r.stderr[-2000:]}")
    timing = json.loads(r.stdout.strip().splitlines()[-1])
    out = {}
    for n in names:
        full = np.fromfile(os.path.join(tmp, f"{n}.bin"))
        out[n] = full_to_plane(cfg, full)
    return out, timing
