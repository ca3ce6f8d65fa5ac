"""mp_field_energy_noalloc: the field energy for callers that cannot allocate
device memory (they own their memory through their own pool or budget, or may
not enter cudaMalloc), computed in the library's fixed scratch array instead of
a context buffer.  Checked through the C ABI against mp_field_energy, the
entry point with context-owned scratch, on two calls in a row with the fields
changed in between.  This file sorts last so that a run stopping at the first
failure has run every other test before it."""
import ctypes as C

import pytest

from mpulse_b200 import abi, runtime
from tests.cases import make_case, random_fields

pytestmark = pytest.mark.gpu

TOL = {abi.MP_FP64: 1e-13, abi.MP_FP32: 1e-12}


def _noalloc_energy(sim):
    ptrs = (C.c_void_p * 6)()
    elem = 0
    for q, n in enumerate(abi.FIELD_NAMES):
        p, count, elem = sim.device_field(n)
        assert count == sim.cfg.field_count()
        ptrs[q] = p
    cfg = sim.cfg
    out = C.c_double()
    rc = runtime.lib().mp_field_energy_noalloc(ptrs, elem, cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz,
                                               None, C.byref(out))
    if rc != abi.MP_OK:
        buf = C.create_string_buffer(256)
        runtime.lib().mp_last_error(None, buf, 256)
        raise runtime.MPulseError(rc, buf.value.decode())
    return out.value


@pytest.mark.parametrize("precision", [abi.MP_FP64, abi.MP_FP32])
def test_noalloc_energy_matches_context_energy_twice(precision):
    cfg = make_case("nonlin_odd_sizes", precision)
    init = random_fields(cfg, seed=41, smooth=True)
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.step(3)
        g.sync()
        first = _noalloc_energy(g)
        want = g.field_energy()
        assert abs(first - want) <= TOL[precision] * abs(want)
        # second call after the fields changed: nothing stale from the first
        g.step(4)
        g.sync()
        second = _noalloc_energy(g)
        want2 = g.field_energy()
        assert abs(second - want2) <= TOL[precision] * abs(want2)
        assert second != first


def test_noalloc_rejects_too_many_planes():
    cfg = make_case("plain_periodic", abi.MP_FP64)
    with runtime.Simulation(cfg) as g:
        ptrs = (C.c_void_p * 6)()
        for q, n in enumerate(abi.FIELD_NAMES):
            ptrs[q] = g.device_field(n)[0]
        out = C.c_double()
        rc = runtime.lib().mp_field_energy_noalloc(ptrs, 8, cfg.nx, cfg.ny, abi.MP_NOALLOC_MAX_PLANES + 1, 1.0, 1.0, 1.0,
                                                   None, C.byref(out))
        assert rc == abi.MP_ERR_INVALID
        buf = C.create_string_buffer(256)
        runtime.lib().mp_last_error(None, buf, 256)
        assert b"exceeds" in buf.value


def test_noalloc_rejects_host_pointers():
    """A host buffer in fields[] is turned into MP_ERR_INVALID on the host,
    before any kernel is launched (nothing reaches the GPU)."""
    import numpy as np
    cfg = make_case("plain_periodic", abi.MP_FP64)
    host = np.zeros(cfg.field_count())
    with runtime.Simulation(cfg) as g:
        ptrs = (C.c_void_p * 6)()
        for q, n in enumerate(abi.FIELD_NAMES):
            ptrs[q] = g.device_field(n)[0]
        ptrs[4] = host.ctypes.data
        out = C.c_double()
        rc = runtime.lib().mp_field_energy_noalloc(ptrs, 8, cfg.nx, cfg.ny, cfg.nz, 1.0, 1.0, 1.0, None,
                                                   C.byref(out))
        assert rc == abi.MP_ERR_INVALID
        buf = C.create_string_buffer(256)
        runtime.lib().mp_last_error(None, buf, 256)
        assert b"fields[4]" in buf.value
        # the library stays usable: a valid call right after it succeeds
        ptrs[4] = g.device_field("By")[0]
        assert _noalloc_energy(g) == pytest.approx(g.field_energy(), rel=1e-13, abs=0.0)
