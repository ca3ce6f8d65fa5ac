"""Field initialisers (pulse_init, gauss_init, wave_init) and FollowMax.

CPU: the oracle's initialisers reproduce the reference build bit for bit (run
with the same setup-file block and no steps), and its FollowMax reproduces a
plain restatement of followmax.cpp:73-113.  GPU: mp_initialize and
mp_follow_max against the oracle."""
import math
import os

import numpy as np
import pytest

from mpulse_b200 import abi
from oracle import pyoracle
from tests.cases import make_case, random_fields, rel_l2


def init_cases():
    out = []
    q = abi.default_init(abi.MP_INIT_PULSE)
    q.k[2] = 2 * math.pi / 0.8
    q.r0, q.z0, q.zc, q.C = 0.3, 0.2, 0.5, 0.7
    q.B[:] = (0.3, 1.0, 0.0)
    q.bound = 2
    out.append(("pulse", q))
    q = abi.default_init(abi.MP_INIT_PLANE_GAUSS)
    q.k[:] = (1, 2, 3)
    q.B[:] = (0.2, 1.0, -0.4)
    out.append(("plane_gauss", q))
    q = abi.default_init(abi.MP_INIT_WAVE)
    q.k[:] = (1, -2, 2)
    q.B[:] = (0.5, 1.0, 0.1)
    q.eps = 1.7
    out.append(("wave", q))
    return out


def _cfg():
    cfg = make_case("lin_all_wave_periodic")  # 20 x 12 x 28, CPML all faces, plane wave
    cfg.boundary = abi.MP_BOUNDARY_XY_PERIODIC
    return cfg


@pytest.mark.skipif(not os.path.exists(pyoracle.REF_BIN), reason="reference build not present")
@pytest.mark.parametrize("name,init", init_cases())
def test_oracle_initialisers_reproduce_reference(name, init):
    cfg = _cfg()
    ref, _ = pyoracle.run_reference(cfg, 0, None, inits=pyoracle.init_block(init))
    o = pyoracle.OracleSim(cfg)
    o.initialize(init)
    for n in abi.FIELD_NAMES:
        np.testing.assert_array_equal(o.download(n), ref[n], err_msg=n)


def _follow_max_restated(line, ipos):
    """followmax.cpp:73-113 on a 1-D line with indices 0..n+1 (ghosts at 0, n+1)."""
    n = len(line) - 2
    while True:
        pm, pp = ipos - 1, ipos + 1
        if pm <= 0:
            pm = n
        if pp >= n + 1:
            pp = 1
        mid, left, right = line[ipos], line[pm], line[pp]
        if right > mid:
            ipos = pp
        elif left > mid:
            ipos = pm
        else:
            break
    return ipos, ipos + (left - right) / (2 * (left - 2 * mid + right))


@pytest.mark.parametrize("dim", [0, 1, 2])
def test_oracle_follow_max_restates_followmax(dim):
    cfg = _cfg()
    o = pyoracle.OracleSim(cfg)
    init = random_fields(cfg, seed=8)
    for k, v in init.items():
        o.upload(k, v)
    pos = (7, 5, 11)
    full = pyoracle.plane_to_full(cfg, o.download("Ey"))  # (nx+2, ny+2, nz+2)
    sl = [pos[0], pos[1], pos[2]]
    sl[dim] = slice(None)
    line = full[tuple(sl)]
    for start in (1, 3, (cfg.nx, cfg.ny, cfg.nz)[dim]):
        want = _follow_max_restated(line, start)
        got = o.follow_max("Ey", dim, pos, start)
        assert got[0] == want[0]
        np.testing.assert_equal(got[1], want[1])  # a flat top gives 0/0 = NaN, as in MPulse


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(abi.MP_FP64, 1e-14), (abi.MP_FP32, 1e-6)])
@pytest.mark.parametrize("name,init", init_cases())
def test_gpu_initialisers_match_oracle(name, init, precision, tol):
    from mpulse_b200 import runtime
    cfg = _cfg()
    base = random_fields(cfg, seed=9)  # wave_init adds to the fields
    o = pyoracle.OracleSim(cfg)
    for k, v in base.items():
        o.upload(k, v)
    o.initialize(init)
    cfg.precision = precision
    with runtime.Simulation(cfg) as g:
        for k, v in base.items():
            g.upload(k, v)
        g.initialize(init)
        for n in abi.FIELD_NAMES:
            assert rel_l2(g.download(n), o.download(n)) <= tol, n


@pytest.mark.gpu
def test_gpu_follow_max_tracks_the_pulse_like_the_oracle():
    """A pulse_init pulse running along z: the FollowMax position of Ex on the
    axis, step by step, on the GPU (FP64) and in the oracle."""
    from mpulse_b200 import runtime
    cfg = _cfg()
    cfg.n_sources = 0
    q = abi.default_init(abi.MP_INIT_PULSE)
    q.k[2] = 2 * math.pi / 0.8
    q.r0, q.z0, q.zc, q.C = 1e6, 0.25, 0.5, 0.0
    q.B[:] = (0.0, 1.0, 0.0)
    o = pyoracle.OracleSim(cfg)
    o.initialize(q)
    pos = (10, 6, 12)
    with runtime.Simulation(cfg) as g:
        g.initialize(q)
        ip_g = ip_o = 12
        for _ in range(8):
            assert o.step(1) == abi.MP_OK
            g.step(1)
            ip_o, x_o = o.follow_max("Ex", 2, pos, ip_o)
            ip_g, x_g = g.follow_max("Ex", 2, pos, ip_g)
            assert ip_g == ip_o
            assert abs(x_g - x_o) <= 1e-9
