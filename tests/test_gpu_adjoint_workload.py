"""The adjoint workload at full size (96^3 cells, 10-cell CPML on all faces,
single-pole medium, 32^3 design region with eps_inf ~ U[1, 4], plane-wave
pulse, |E|^2 objective over the 8^3 monitor box, 1500 steps, a checkpoint every
50 steps): the FP64 adjoint gradient dJ/d(eps_inf) and dJ/d(Delta-eps factor)
against FP64 central finite differences (h = 1e-4) of mp_objective at 32
seeded design cells, each within 1e-4 relative."""
import numpy as np
import pytest

from mpulse_b200 import abi, configs, runtime

pytestmark = pytest.mark.gpu

H = 1e-4
TOL = 1e-4
N_PROBES = 32


def _sim(cfg, des):
    g = runtime.Simulation(cfg)
    for k, v in des.items():
        g.upload_design(k, v)
    return g


def test_workload_adjoint_matches_central_differences():
    cfg, des, adj = configs.c4_adjoint(abi.MP_FP64)
    assert (cfg.nx, cfg.ny, cfg.nz, adj.steps, adj.checkpoint_every) == (96, 96, 96, 1500, 50)
    des = dict(des, DesignDepsScale=np.ones_like(des["DesignEps"]))
    with _sim(cfg, des) as g:
        J, grads = g.adjoint(adj)
    rng = np.random.default_rng(4)
    shape = des["DesignEps"].shape
    probes = {tuple(int(rng.integers(0, n)) for n in shape) for _ in range(4 * N_PROBES)}
    probes = sorted(probes)[:N_PROBES]
    assert len(probes) == N_PROBES
    worst = {}
    for name in ("DesignEps", "DesignDepsScale"):
        errs = []
        for idx in probes:
            vals = []
            for sgn in (1.0, -1.0):
                d = {k: v.copy() for k, v in des.items()}
                d[name][idx] += sgn * H
                with _sim(cfg, d) as g:
                    vals.append(g.objective(adj))
            fd = (vals[0] - vals[1]) / (2 * H)
            errs.append(abs(fd - grads[name][idx]) / abs(fd))
            assert abs(fd - grads[name][idx]) <= TOL * abs(fd), (name, idx, fd, grads[name][idx], J)
        worst[name] = max(errs)
    print("max relative error at the probe cells:", worst)
