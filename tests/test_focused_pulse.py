"""focused_pulse_inject: MPulse's plug-in (focusedpulseinject.cpp) does not
compile, so the pulse is defined here as the paraxial short-pulse closed form
(shortpulseinject.cpp) with the same keys.  Parity is therefore unpinned against
the reference; what is checked is that the kind runs that closed form in the
oracle and on the GPU."""
import numpy as np
import pytest

from mpulse_b200 import abi
from oracle import pyoracle
from tests.cases import make_case, random_fields


def _pair():
    short = make_case("nonlin_all_short")
    focused = make_case("nonlin_all_short")
    focused.sources[0].kind = abi.MP_SOURCE_FOCUSED_PULSE
    return short, focused


def test_oracle_focused_pulse_is_the_short_pulse_closed_form():
    short, focused = _pair()
    init = random_fields(short, seed=3)
    out = []
    for cfg in (short, focused):
        o = pyoracle.OracleSim(cfg)
        for n, v in init.items():
            o.upload(n, v)
        assert o.step(12) == abi.MP_OK
        out.append({n: o.download(n) for n in abi.FIELD_NAMES})
    for n in abi.FIELD_NAMES:
        np.testing.assert_array_equal(out[0][n], out[1][n])


@pytest.mark.gpu
def test_gpu_focused_pulse_is_the_short_pulse_closed_form():
    from mpulse_b200 import runtime
    short, focused = _pair()
    init = random_fields(short, seed=4)
    out = []
    for cfg in (short, focused):
        with runtime.Simulation(cfg) as g:
            for n, v in init.items():
                g.upload(n, v)
            g.step(12)
            out.append({n: g.download(n) for n in abi.FIELD_NAMES})
    for n in abi.FIELD_NAMES:
        np.testing.assert_array_equal(out[0][n], out[1][n])
