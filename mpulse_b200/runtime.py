"""ctypes binding of the C ABI in include/mpulse_b200.h (libmpulse_b200.so).

``Simulation`` is a thin object wrapper over one ``mp_ctx``: the host-side
counterpart of MPulse's FieldSimulation + FieldSolver pair for the
time-stepping path (src/fieldsim.cpp:31-112, src/fieldsolver.h:10-37).  There is
no CPU fallback: if the library is missing or no GPU is present, creating a
Simulation raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
# MPULSE_B200_LIB selects another build of the library (e.g. a tuning variant).
LIB_PATH = os.environ.get("MPULSE_B200_LIB") or os.path.join(HERE, "libmpulse_b200.so")

# Every entry point include/mpulse_b200.h declares.
EXPORTED = (
    "mp_config_defaults", "mp_create", "mp_destroy", "mp_set_stream", "mp_field_size",
    "mp_upload", "mp_download", "mp_step", "mp_step_async", "mp_check_status",
    "mp_get_time", "mp_set_time", "mp_sync", "mp_device_field", "mp_launch_count",
    "mp_last_error", "mp_create_error", "mp_kernel_times", "mp_field_energy",
    "mp_field_energy_noalloc", "mp_objective", "mp_adjoint", "mp_objective_record", "mp_adjoint_reverse",
    "mp_release_record", "mp_set_host_checkpoint_budget", "mp_state_size", "mp_save_state",
    "mp_load_state", "mp_init_defaults", "mp_initialize", "mp_follow_max", "mp_kerr_counts",
    "mp_diag_file_name", "mp_hdf5_create", "mp_hdf5_write_field", "mp_hdf5_write_slice", "mp_hdf5_write_grid", "mp_hdf5_close",
)

_lib = None


class MPulseError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Loads libmpulse_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mpulse_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, cp, sz, dp = C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_double)
    L.mp_config_defaults.argtypes = [C.POINTER(abi.Config)]
    L.mp_config_defaults.restype = None
    L.mp_create.argtypes = [C.POINTER(abi.Config), C.POINTER(vp)]
    L.mp_create.restype = C.c_int
    L.mp_destroy.argtypes = [vp]
    L.mp_destroy.restype = None
    L.mp_set_stream.argtypes = [vp, vp]
    L.mp_set_stream.restype = C.c_int
    L.mp_field_size.argtypes = [vp, cp, C.POINTER(sz)]
    L.mp_field_size.restype = C.c_int
    L.mp_upload.argtypes = [vp, cp, dp, sz]
    L.mp_upload.restype = C.c_int
    L.mp_download.argtypes = [vp, cp, dp, sz]
    L.mp_download.restype = C.c_int
    for f in (L.mp_step, L.mp_step_async):
        f.argtypes = [vp, C.c_int]
        f.restype = C.c_int
    L.mp_check_status.argtypes = [vp]
    L.mp_check_status.restype = C.c_int
    L.mp_get_time.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.mp_get_time.restype = C.c_int
    L.mp_set_time.argtypes = [vp, C.c_longlong]
    L.mp_set_time.restype = C.c_int
    L.mp_sync.argtypes = [vp]
    L.mp_sync.restype = C.c_int
    L.mp_device_field.argtypes = [vp, cp, C.POINTER(vp), C.POINTER(sz), C.POINTER(C.c_int)]
    L.mp_device_field.restype = C.c_int
    L.mp_launch_count.argtypes = [vp]
    L.mp_launch_count.restype = C.c_longlong
    L.mp_last_error.argtypes = [vp, C.c_char_p, sz]
    L.mp_last_error.restype = C.c_int
    L.mp_kernel_times.argtypes = [vp, C.c_int, dp, dp, dp]
    L.mp_kernel_times.restype = C.c_int
    L.mp_field_energy.argtypes = [vp, dp]
    L.mp_field_energy.restype = C.c_int
    L.mp_field_energy_noalloc.argtypes = [C.POINTER(vp), C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                          C.c_double, C.c_double, vp, dp]
    L.mp_field_energy_noalloc.restype = C.c_int
    L.mp_objective.argtypes = [vp, C.POINTER(abi.AdjointConfig), dp]
    L.mp_objective.restype = C.c_int
    L.mp_adjoint.argtypes = [vp, C.POINTER(abi.AdjointConfig), dp, dp, dp, dp]
    L.mp_adjoint.restype = C.c_int
    L.mp_objective_record.argtypes = [vp, C.POINTER(abi.AdjointConfig), dp]
    L.mp_objective_record.restype = C.c_int
    L.mp_adjoint_reverse.argtypes = [vp, dp, dp, dp, dp]
    L.mp_adjoint_reverse.restype = C.c_int
    L.mp_release_record.argtypes = [vp]
    L.mp_release_record.restype = C.c_int
    L.mp_set_host_checkpoint_budget.argtypes = [vp, C.c_double]
    L.mp_set_host_checkpoint_budget.restype = C.c_int
    L.mp_state_size.argtypes = [vp, C.POINTER(sz)]
    L.mp_state_size.restype = C.c_int
    L.mp_save_state.argtypes = [vp, vp, sz]
    L.mp_save_state.restype = C.c_int
    L.mp_load_state.argtypes = [vp, vp, sz]
    L.mp_load_state.restype = C.c_int
    L.mp_init_defaults.argtypes = [C.c_int, C.POINTER(abi.Init)]
    L.mp_init_defaults.restype = None
    L.mp_initialize.argtypes = [vp, C.POINTER(abi.Init)]
    L.mp_initialize.restype = C.c_int
    L.mp_follow_max.argtypes = [vp, cp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), dp]
    L.mp_follow_max.restype = C.c_int
    L.mp_kerr_counts.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    L.mp_kerr_counts.restype = C.c_int
    L.mp_diag_file_name.argtypes = [cp, C.c_int, C.c_longlong, C.c_char_p, sz]
    L.mp_diag_file_name.restype = C.c_int
    L.mp_hdf5_create.argtypes = [cp, C.c_int, C.c_longlong, C.POINTER(vp)]
    L.mp_hdf5_create.restype = C.c_int
    L.mp_hdf5_write_field.argtypes = [vp, vp, cp]
    L.mp_hdf5_write_field.restype = C.c_int
    L.mp_hdf5_write_slice.argtypes = [vp, vp, cp, C.c_int, C.c_int]
    L.mp_hdf5_write_slice.restype = C.c_int
    L.mp_hdf5_write_grid.argtypes = [vp, dp, C.POINTER(sz)]
    L.mp_hdf5_write_grid.restype = C.c_int
    L.mp_hdf5_close.argtypes = [vp]
    L.mp_hdf5_close.restype = C.c_int
    L.mp_create_error.argtypes = []
    L.mp_create_error.restype = C.c_char_p
    _lib = L
    return L


def _global_error() -> str:
    buf = C.create_string_buffer(512)
    lib().mp_last_error(None, buf, 512)
    return buf.value.decode()


def diag_file_name(pattern: str, proc_id: int, time: int) -> str:
    """DiagnosticInterface::parsedFileName (diagnostic.cpp:52-70) through
    mp_diag_file_name."""
    out = C.create_string_buffer(len(pattern) + 64)
    rc = lib().mp_diag_file_name(pattern.encode(), proc_id, time, out, len(out))
    if rc != abi.MP_OK:
        raise MPulseError(rc, _global_error())
    return out.value.decode()


class Hdf5File:
    """One HDF5 output file (mp_hdf5_create ... mp_hdf5_close), the file of
    an HDFostream: datasets "data0", "data1", ... in the order written."""

    def __init__(self, pattern: str, proc_id: int = 0, time: int = 0):
        self.name = diag_file_name(pattern, proc_id, time)
        self._h = C.c_void_p()
        rc = lib().mp_hdf5_create(pattern.encode(), proc_id, time, C.byref(self._h))
        if rc != abi.MP_OK:
            raise MPulseError(rc, _global_error())

    def write_field(self, sim: "Simulation", name: str):
        """FieldDiag::write: the field `name` of sim as the next dataset."""
        rc = lib().mp_hdf5_write_field(self._h, sim._h, name.encode())
        if rc != abi.MP_OK:
            raise MPulseError(rc, sim.last_error() or _global_error())

    def write_slice(self, sim: "Simulation", name: str, plane: str, pos: int):
        """FieldSliceDiag::write: the plane ("x", "y" or "z") of field `name`
        through MPulse index pos as the next dataset (nothing when pos is not
        strictly inside the grid)."""
        rc = lib().mp_hdf5_write_slice(self._h, sim._h, name.encode(), "xyz".index(plane), int(pos))
        if rc != abi.MP_OK:
            raise MPulseError(rc, sim.last_error() or _global_error())

    def write_grid(self, a):
        """A 3-D host array (C order) as the next dataset."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        dims = (C.c_size_t * 3)(*a.shape)
        rc = lib().mp_hdf5_write_grid(self._h, _dptr(a), dims)
        if rc != abi.MP_OK:
            raise MPulseError(rc, _global_error())

    def close(self):
        if self._h:
            rc = lib().mp_hdf5_close(self._h)
            self._h = None
            if rc != abi.MP_OK:
                raise MPulseError(rc, _global_error())

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def write_hdf5_arrays(pattern: str, arrays, proc_id: int = 0, time: int = 0) -> str:
    """Writes 3-D host arrays (C order) as the datasets "data0", "data1", ...
    of one HDF5 file (mp_hdf5_write_grid); returns the file name."""
    with Hdf5File(pattern, proc_id, time) as f:
        for a in arrays:
            f.write_grid(a)
    return f.name


def library_defaults() -> abi.Config:
    c = abi.Config()
    lib().mp_config_defaults(C.byref(c))
    return c


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Simulation:
    """One simulation held in HBM (an ``mp_ctx``)."""

    def __init__(self, cfg: abi.Config):
        L = lib()
        self.cfg = cfg
        h = C.c_void_p()
        rc = L.mp_create(C.byref(cfg), C.byref(h))
        if rc != abi.MP_OK:
            raise MPulseError(rc, L.mp_create_error().decode())
        self._h = h

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None):
            lib().mp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- errors
    def last_error(self) -> str:
        buf = C.create_string_buffer(512)
        lib().mp_last_error(self._h, buf, 512)
        return buf.value.decode()

    def _check(self, rc: int):
        if rc != abi.MP_OK:
            raise MPulseError(rc, self.last_error())

    # -- fields
    def upload(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        self._check(lib().mp_upload(self._h, name.encode(), _dptr(a), a.size))

    def download(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.cfg.field_count(), dtype=np.float64)
        self._check(lib().mp_download(self._h, name.encode(), _dptr(out), out.size))
        return out.reshape(self.cfg.field_shape())

    def device_field(self, name: str):
        p, n, es = C.c_void_p(), C.c_size_t(), C.c_int()
        self._check(lib().mp_device_field(self._h, name.encode(), C.byref(p), C.byref(n), C.byref(es)))
        return p.value, n.value, es.value

    # -- stepping
    def step(self, n: int = 1):
        self._check(lib().mp_step(self._h, int(n)))

    def step_async(self, n: int = 1):
        self._check(lib().mp_step_async(self._h, int(n)))

    def check_status(self):
        self._check(lib().mp_check_status(self._h))

    def sync(self):
        self._check(lib().mp_sync(self._h))

    def set_stream(self, stream_ptr: int | None):
        self._check(lib().mp_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    @property
    def time(self) -> int:
        t = C.c_longlong()
        self._check(lib().mp_get_time(self._h, C.byref(t)))
        return t.value

    @time.setter
    def time(self, t: int):
        self._check(lib().mp_set_time(self._h, int(t)))

    def kernel_times(self, n: int) -> dict:
        """Runs n steps with per-kernel CUDA-event timing; average ms per launch."""
        e, b, s = C.c_double(), C.c_double(), C.c_double()
        self._check(lib().mp_kernel_times(self._h, int(n), C.byref(e), C.byref(b), C.byref(s)))
        return {"e_half_ms": e.value, "b_half_ms": b.value, "sources_ms": s.value}

    def kerr_counts(self) -> tuple[int, int]:
        """(Kerr solves, Newton iterations) of the E half-steps since the last
        call (mp_kerr_counts); resets the device counters."""
        a, b = C.c_longlong(), C.c_longlong()
        self._check(lib().mp_kerr_counts(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def field_energy(self) -> float:
        """FieldEnergyDiag::calculate (fielddiag.cpp:255-286) on the device state."""
        e = C.c_double()
        self._check(lib().mp_field_energy(self._h, C.byref(e)))
        return e.value

    @property
    def launches(self) -> int:
        return lib().mp_launch_count(self._h)

    # -- design region, objective, adjoint
    def upload_design(self, name: str, arr):
        """One of abi.DESIGN_NAMES, shaped like abi.design_shape(cfg)."""
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        self._check(lib().mp_upload(self._h, name.encode(), _dptr(a), a.size))

    def download_design(self, name: str) -> np.ndarray:
        shape = abi.design_shape(self.cfg)
        out = np.empty(int(np.prod(shape)), dtype=np.float64)
        self._check(lib().mp_download(self._h, name.encode(), _dptr(out), out.size))
        return out.reshape(shape)

    def objective(self, adj: abi.AdjointConfig) -> float:
        """Runs adj.steps steps and returns the objective J (mp_objective)."""
        J = C.c_double()
        self._check(lib().mp_objective(self._h, C.byref(adj), C.byref(J)))
        return J.value

    def set_host_checkpoint_budget(self, nbytes: float):
        """Pinned host memory mp_adjoint may use for checkpoints
        (mp_set_host_checkpoint_budget)."""
        self._check(lib().mp_set_host_checkpoint_budget(self._h, float(nbytes)))

    def adjoint(self, adj: abi.AdjointConfig) -> tuple[float, dict]:
        """J and its gradient with respect to the design maps (mp_adjoint):
        {"DesignEps": .., "DesignDepsScale": .., "DesignChiScale": ..}."""
        shape = abi.design_shape(self.cfg)
        if shape is None:  # no design box: the library rejects the call
            J = C.c_double()
            self._check(lib().mp_adjoint(self._h, C.byref(adj), C.byref(J), None, None, None))
            return J.value, {}
        n = int(np.prod(shape))
        g = [np.empty(n) for _ in range(3)]
        J = C.c_double()
        self._check(lib().mp_adjoint(self._h, C.byref(adj), C.byref(J), _dptr(g[0]), _dptr(g[1]), _dptr(g[2])))
        return J.value, {name: a.reshape(shape) for name, a in zip(abi.DESIGN_NAMES, g)}

    def objective_record(self, adj: abi.AdjointConfig) -> float:
        """The forward part of adjoint(adj): runs the steps, returns J and
        keeps the checkpoints for adjoint_reverse (mp_objective_record)."""
        J = C.c_double()
        self._check(lib().mp_objective_record(self._h, C.byref(adj), C.byref(J)))
        return J.value

    def adjoint_reverse(self) -> tuple[float, dict]:
        """J and the gradient of the run objective_record recorded
        (mp_adjoint_reverse); the record is released."""
        shape = abi.design_shape(self.cfg)
        J = C.c_double()
        if shape is None:
            self._check(lib().mp_adjoint_reverse(self._h, C.byref(J), None, None, None))
            return J.value, {}
        n = int(np.prod(shape))
        g = [np.empty(n) for _ in range(3)]
        self._check(lib().mp_adjoint_reverse(self._h, C.byref(J), _dptr(g[0]), _dptr(g[1]), _dptr(g[2])))
        return J.value, {name: a.reshape(shape) for name, a in zip(abi.DESIGN_NAMES, g)}

    def release_record(self):
        """Frees what objective_record kept (mp_release_record)."""
        self._check(lib().mp_release_record(self._h))

    # -- HDF5 field dumps (FieldDiag through HDFostream)
    def write_hdf5(self, pattern: str, fields, proc_id: int = 0, time: int | None = None) -> str:
        """Writes `fields` of the device state to one HDF5 file named by
        `pattern` after the #p / #t substitution with proc_id and time (the
        context's time by default); returns the file name."""
        time = self.time if time is None else time
        with Hdf5File(pattern, proc_id, time) as f:
            for n in fields:
                f.write_field(self, n)
        return f.name

    # -- checkpoint / restart
    def save_state(self) -> bytes:
        """The whole device state and the time (mp_save_state)."""
        n = C.c_size_t()
        self._check(lib().mp_state_size(self._h, C.byref(n)))
        buf = (C.c_char * n.value)()
        self._check(lib().mp_save_state(self._h, buf, n.value))
        return bytes(buf)

    def load_state(self, data: bytes):
        buf = C.create_string_buffer(data, len(data))
        self._check(lib().mp_load_state(self._h, buf, len(data)))

    # -- initialisers and FollowMax
    def initialize(self, init: abi.Init):
        """pulse_init / gauss_init / wave_init on the device (mp_initialize)."""
        self._check(lib().mp_initialize(self._h, C.byref(init)))

    def follow_max(self, field: str, dim: int, pos, ipos: int) -> tuple[int, float]:
        """FollowMax::calculate from integer position ipos along dim through
        MPulse cell pos: (new integer position, interpolated position)."""
        p = (C.c_int * 3)(*pos)
        ip = C.c_int(ipos)
        out = C.c_double()
        self._check(lib().mp_follow_max(self._h, field.encode(), dim, p, C.byref(ip), C.byref(out)))
        return ip.value, out.value
