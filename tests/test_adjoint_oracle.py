"""The adjoint's restatement on the CPU (oracle/pyadjoint.py) against the C
oracle: its forward step reproduces the oracle's (design maps included), its
reverse step is the exact transpose of the linear step (dot-product test),
and the gradients it assembles match central finite differences of the
oracle's objective.  These pin the arithmetic that mp_adjoint's kernels are
checked against in test_gpu_adjoint.py."""
import copy
import math

import numpy as np
import pytest

from mpulse_b200 import abi, configs
from oracle import pyadjoint, pyoracle
from tests.cases import random_fields, rel_l2


def design_case(solver, cpml, n=(10, 8, 14), source=False):
    c = configs.base(*n, courant=configs.MEDIUM_COURANT)
    c.solver = solver
    c.boundary = abi.MP_BOUNDARY_XY_PERIODIC
    for k, p in enumerate(configs.SILICA_POLES):
        c.poles[k].eps, c.poles[k].delta, c.poles[k].om2 = p
    c.poles[2].eps, c.poles[2].delta, c.poles[2].om2 = 0.0, 0.0, 1.0
    c.medium_z0, c.medium_z1 = 4, n[2] + 1
    c.eps_bg = 1.1
    c.chi = 0.3
    c.cpml = cpml
    c.cpml_d = 3
    c.cpml_kappa_max = 2.0
    c.cpml_a_max = 0.1
    c.cpml_sigma_max = 40.0
    c.design_box[:] = (3, 7, 2, 6, 6, 10)
    if source:
        c.n_sources = 1
        s = c.sources[0]
        s.kind = abi.MP_SOURCE_PLANE_GAUSS
        s.distance = 3
        s.k[:] = (0.0, 0.0, 2 * math.pi / 0.8)
        s.H[:] = (0.0, 1.0, 0.0)
        s.width = 2.0
        s.offset = 3.0
    return c


def design_maps(cfg, seed):
    rng = np.random.default_rng(seed)
    ds = abi.design_shape(cfg)
    return {"DesignEps": rng.uniform(1, 4, ds), "DesignDepsScale": rng.uniform(0.5, 1.5, ds),
            "DesignChiScale": rng.uniform(0.5, 1.5, ds)}


def clean_init(cfg, seed, smooth=False, scale=0.3):
    """Random fields with the xy-periodic boundary's fixed ghost planes at zero."""
    init = random_fields(cfg, seed=seed, scale=scale, smooth=smooth)
    for n in ("Ex", "Ey", "Ez"):
        init[n][0] = 0
        init[n][-1] = 0
    for n in ("Bx", "By", "Bz"):
        init[n][-1] = 0
    return init


@pytest.mark.parametrize("solver", [abi.MP_SOLVER_PLRC_LIN, abi.MP_SOLVER_PLRC_NONLIN])
@pytest.mark.parametrize("cpml", [abi.MP_CPML_ALL, abi.MP_CPML_Z])
def test_restated_forward_matches_oracle(solver, cpml):
    cfg = design_case(solver, cpml)
    des = design_maps(cfg, 1)
    init = clean_init(cfg, 3)
    o = pyoracle.OracleSim(cfg)
    for k, v in init.items():
        o.upload(k, v)
    for k, v in des.items():
        o.upload_design(k, v)
    assert o.step(6) == abi.MP_OK
    m = pyadjoint.Model(cfg)
    m.set_design(des["DesignEps"], des["DesignDepsScale"], des["DesignChiScale"])
    st = m.zero_state()
    for c, name in enumerate(abi.FIELD_NAMES):
        (st["E"] if c < 3 else st["B"])[c % 3][:] = init[name]
    for _ in range(6):
        m.step(st)
    for c, name in enumerate(abi.FIELD_NAMES):
        got = (st["E"] if c < 3 else st["B"])[c % 3]
        assert rel_l2(got, o.download(name)) <= 1e-13, name


def _inner(a, b):
    t = 0.0
    for c in range(3):
        t += np.sum(a["E"][c] * b["E"][c]) + np.sum(a["B"][c] * b["B"][c])
    for n in range(len(a["psi"])):
        for c in range(3):
            t += np.sum((np.conj(a["psi"][n][c]) * b["psi"][n][c]).real)
    for key in ("psiE", "psiH"):
        for l in range(len(a[key])):
            for q in range(2):
                t += np.sum(a[key][l][q] * b[key][l][q])
    return t


def _random_state(m, rng):
    st = m.zero_state()
    for c in range(3):
        st["E"][c][:] = np.where(m.ecell, rng.standard_normal(m.shape), 0)
        st["B"][c][:] = np.where(m.bcell, rng.standard_normal(m.shape), 0)
    for n in range(len(st["psi"])):
        for c in range(3):
            st["psi"][n][c][:] = np.where(m.med, rng.standard_normal(m.shape) + 1j * rng.standard_normal(m.shape), 0)
    for key, cells in (("psiE", m.ecell), ("psiH", m.bcell)):
        for l, (_dim, mask, _b, _c) in enumerate(m.layers[0 if key == "psiE" else 1]):
            for q in range(2):
                st[key][l][q][:] = np.where(mask & cells, rng.standard_normal(m.shape), 0)
    return st


@pytest.mark.parametrize("cpml", [abi.MP_CPML_ALL, abi.MP_CPML_Z])
def test_reverse_step_is_the_transpose_of_the_linear_step(cpml):
    """<M x, y> = <x, M^T y> for the linear PLRC step with CPML and design maps."""
    rng = np.random.default_rng(7)
    cfg = design_case(abi.MP_SOLVER_PLRC_LIN, cpml)
    m = pyadjoint.Model(cfg)
    des = design_maps(cfg, 2)
    m.set_design(des["DesignEps"], des["DesignDepsScale"])
    x = _random_state(m, rng)
    y = _random_state(m, rng)
    Mx = m.step(copy.deepcopy(x))
    lhs = _inner(Mx, y)
    MTy = m.reverse_step([e.copy() for e in x["E"]], Mx["E"], copy.deepcopy(y))
    rhs = _inner(x, MTy)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("solver,kind", [(abi.MP_SOLVER_PLRC_LIN, abi.MP_OBJ_E2_BOX),
                                         (abi.MP_SOLVER_PLRC_NONLIN, abi.MP_OBJ_SZ_PLANE),
                                         (abi.MP_SOLVER_PLRC_NONLIN, abi.MP_OBJ_E2_BOX)])
def test_restated_gradient_matches_finite_differences(solver, kind):
    cfg = design_case(solver, abi.MP_CPML_ALL, source=True)
    des = design_maps(cfg, 5)
    init = clean_init(cfg, 4, smooth=True, scale=0.2)
    box = (4, 7, 3, 6, 11, 13) if kind == abi.MP_OBJ_E2_BOX else (1, 10, 1, 8, 12, 12)
    adj = abi.adjoint_config(kind, box, 12)
    J, grad = pyadjoint.adjoint_gradient(cfg, adj, init, des)

    def objective(d):
        o = pyoracle.OracleSim(cfg)
        for k, v in init.items():
            o.upload(k, v)
        for k, v in d.items():
            o.upload_design(k, v)
        return o.objective(adj)

    assert abs(J - objective(des)) <= 1e-13 * abs(J)
    rng = np.random.default_rng(9)
    names = (("DesignEps", "eps"), ("DesignDepsScale", "s"))
    if solver == abi.MP_SOLVER_PLRC_NONLIN:
        names += (("DesignChiScale", "u"),)
    for name, key in names:
        scale = np.max(np.abs(grad[key]))
        for _ in range(2):
            idx = tuple(int(rng.integers(0, n)) for n in grad[key].shape)
            h = 1e-5
            dp = {k: v.copy() for k, v in des.items()}
            dm = {k: v.copy() for k, v in des.items()}
            dp[name][idx] += h
            dm[name][idx] -= h
            fd = (objective(dp) - objective(dm)) / (2 * h)
            assert abs(fd - grad[key][idx]) <= 1e-6 * scale + 1e-4 * abs(fd), (name, idx, fd, grad[key][idx])
