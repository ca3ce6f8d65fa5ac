"""mp_objective and mp_adjoint on the GPU against the CPU restatement
(oracle/pyadjoint.py, itself checked against finite differences of the C oracle
in test_adjoint_oracle.py), against central finite differences of the GPU's
own FP64 forward, FP32 against FP64, and through torch.autograd."""
import numpy as np
import pytest
import torch

from mpulse_b200 import abi, adjoint, runtime
from oracle import pyadjoint, pyoracle
from tests.cases import rel_l2
from tests.test_adjoint_oracle import clean_init, design_case, design_maps

pytestmark = pytest.mark.gpu

BOXES = {abi.MP_OBJ_E2_BOX: (4, 7, 3, 6, 11, 13), abi.MP_OBJ_SZ_PLANE: (1, 10, 1, 8, 12, 12)}


def gpu_sim(cfg, init, des):
    g = runtime.Simulation(cfg)
    for k, v in init.items():
        g.upload(k, v)
    for k, v in des.items():
        g.upload_design(k, v)
    return g


@pytest.mark.parametrize("precision,tol", [(abi.MP_FP64, 1e-12), (abi.MP_FP32, 1e-5)])
@pytest.mark.parametrize("solver", [abi.MP_SOLVER_PLRC_LIN, abi.MP_SOLVER_PLRC_NONLIN])
def test_forward_with_design_maps_matches_oracle(solver, precision, tol):
    cfg = design_case(solver, abi.MP_CPML_ALL, source=True)
    des = design_maps(cfg, 11)
    init = clean_init(cfg, 12, smooth=True)
    o = pyoracle.OracleSim(cfg)
    for k, v in init.items():
        o.upload(k, v)
    for k, v in des.items():
        o.upload_design(k, v)
    assert o.step(20) == abi.MP_OK
    cfg.precision = precision
    with gpu_sim(cfg, init, des) as g:
        for k, v in des.items():
            np.testing.assert_array_equal(g.download_design(k), v)
        g.step(20)
        for n in abi.FIELD_NAMES:
            assert rel_l2(g.download(n), o.download(n)) <= tol, n


def test_default_design_maps_change_nothing():
    """A design box with eps_inf = eps and factors 1 steps bit for bit like no box."""
    cfg = design_case(abi.MP_SOLVER_PLRC_NONLIN, abi.MP_CPML_Z, source=True)
    init = clean_init(cfg, 13)
    plain = design_case(abi.MP_SOLVER_PLRC_NONLIN, abi.MP_CPML_Z, source=True)
    plain.design_box[:] = (1, 0, 1, 0, 1, 0)
    with gpu_sim(cfg, init, {}) as a, gpu_sim(plain, init, {}) as b:
        a.step(15)
        b.step(15)
        for n in abi.FIELD_NAMES:
            np.testing.assert_array_equal(a.download(n), b.download(n))


@pytest.mark.parametrize("kind", [abi.MP_OBJ_E2_BOX, abi.MP_OBJ_SZ_PLANE])
def test_objective_matches_oracle(kind):
    cfg = design_case(abi.MP_SOLVER_PLRC_NONLIN, abi.MP_CPML_ALL, source=True)
    des = design_maps(cfg, 14)
    init = clean_init(cfg, 15, smooth=True, scale=0.2)
    adj = abi.adjoint_config(kind, BOXES[kind], 16)
    o = pyoracle.OracleSim(cfg)
    for k, v in init.items():
        o.upload(k, v)
    for k, v in des.items():
        o.upload_design(k, v)
    want = o.objective(adj)
    with gpu_sim(cfg, init, des) as g:
        got = g.objective(adj)
        assert g.time == 16
    assert abs(got - want) <= 1e-12 * abs(want)


@pytest.mark.parametrize("solver", [abi.MP_SOLVER_PLRC_LIN, abi.MP_SOLVER_PLRC_NONLIN])
@pytest.mark.parametrize("kind", [abi.MP_OBJ_E2_BOX, abi.MP_OBJ_SZ_PLANE])
@pytest.mark.parametrize("every", [0, 5, 8])
def test_fp64_adjoint_matches_restatement(solver, kind, every):
    """checkpoint_every 0 keeps the whole history from the forward run; 5
    recomputes the segment [0,5) from its checkpoint ([5,10) keeps its history
    from the first run); 8 has two segments, the first kept from the first
    run."""
    cfg = design_case(solver, abi.MP_CPML_ALL, source=True)
    des = design_maps(cfg, 16)
    init = clean_init(cfg, 17, smooth=True, scale=0.2)
    adj = abi.adjoint_config(kind, BOXES[kind], 12, checkpoint_every=every)
    J_ref, g_ref = pyadjoint.adjoint_gradient(cfg, adj, init, des)
    with gpu_sim(cfg, init, des) as g:
        J, grads = g.adjoint(adj)
        assert g.time == 12
        # the state ends as after the forward run
        o = pyoracle.OracleSim(cfg)
        for k, v in init.items():
            o.upload(k, v)
        for k, v in des.items():
            o.upload_design(k, v)
        o.step(12)
        for n in abi.FIELD_NAMES:
            assert rel_l2(g.download(n), o.download(n)) <= 1e-12, n
    assert abs(J - J_ref) <= 1e-12 * abs(J_ref)
    for name, key in (("DesignEps", "eps"), ("DesignDepsScale", "s"), ("DesignChiScale", "u")):
        ref = g_ref[key]
        if not np.any(ref):
            assert not np.any(grads[name]), name
            continue
        assert rel_l2(grads[name], ref) <= 1e-10, (name, rel_l2(grads[name], ref))


@pytest.mark.parametrize("per_cell", [864.0, 648.0, 516.0])
def test_adjoint_memory_budget_schedule(per_cell):
    """Budgets that hold only a few states give the same J and gradient as the
    whole history: one state is about 8 B x cells x (6 fields + 2 poles x 3
    components x 2 x 11/16 medium planes) plus the CPML psi (~126 B per cell),
    one step of history 24 B per cell.  864 B per cell: two checkpoints; 648:
    three slots for six chunks (binomial placement, chunks run up to three
    times); 516: one slot, every chunk run again from the start."""
    cfg = design_case(abi.MP_SOLVER_PLRC_LIN, abi.MP_CPML_Z, source=True)
    des = design_maps(cfg, 18)
    init = clean_init(cfg, 19, smooth=True, scale=0.2)
    full = abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], 30)
    with gpu_sim(cfg, init, des) as g:
        J0, g0 = g.adjoint(full)
    tight = abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], 30,
                               mem_budget=per_cell * cfg.field_count())
    with gpu_sim(cfg, init, des) as g:
        J1, g1 = g.adjoint(tight)
        assert g.time == 30
    assert abs(J1 - J0) <= 1e-14 * abs(J0)
    for name in abi.DESIGN_NAMES[:2]:
        assert rel_l2(g1[name], g0[name]) <= 1e-13


@pytest.mark.parametrize("steps", [30, 47])
def test_adjoint_host_checkpoints(steps):
    """A device budget of one state slot (every chunk run again from the start)
    with room for segment checkpoints in host memory: the two-level schedule
    runs fewer kernels and gives the same J and gradient as the whole history
    (the recomputed forward steps are the same arithmetic)."""
    cfg = design_case(abi.MP_SOLVER_PLRC_LIN, abi.MP_CPML_Z, source=True)
    des = design_maps(cfg, 22)
    init = clean_init(cfg, 23, smooth=True, scale=0.2)
    full = abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], steps)
    with gpu_sim(cfg, init, des) as g:
        J0, g0 = g.adjoint(full)
    tight = abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], steps,
                               mem_budget=516 * cfg.field_count())
    launches = {}
    for nstates in (0, 12):
        with gpu_sim(cfg, init, des) as g:
            g.set_host_checkpoint_budget(nstates * len(g.save_state()))  # a saved state: one state and a header
            l0 = g.launches
            J1, g1 = g.adjoint(tight)
            launches[nstates] = g.launches - l0
            assert g.time == steps
        assert abs(J1 - J0) <= 1e-14 * abs(J0)
        for name in abi.DESIGN_NAMES[:2]:
            assert rel_l2(g1[name], g0[name]) <= 1e-13
    assert launches[12] < launches[0], launches


def test_host_checkpoint_budget_rejects_bad_values():
    cfg = design_case(abi.MP_SOLVER_PLRC_LIN, abi.MP_CPML_Z, source=True)
    with gpu_sim(cfg, {}, {}) as g:
        for bad in (-1.0, float("nan"), float("inf")):
            with pytest.raises(runtime.MPulseError):
                g.set_host_checkpoint_budget(bad)


def test_adjoint_memory_budget_too_small():
    cfg = design_case(abi.MP_SOLVER_PLRC_LIN, abi.MP_CPML_Z, source=True)
    with gpu_sim(cfg, {}, {}) as g:
        with pytest.raises(runtime.MPulseError):
            g.adjoint(abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], 30, mem_budget=1000.0))


def test_fp32_adjoint_matches_fp64():
    cfg = design_case(abi.MP_SOLVER_PLRC_NONLIN, abi.MP_CPML_ALL, source=True)
    des = design_maps(cfg, 20)
    init = clean_init(cfg, 21, smooth=True, scale=0.2)
    adj = abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], 20)
    with gpu_sim(cfg, init, des) as g:
        J64, g64 = g.adjoint(adj)
    cfg.precision = abi.MP_FP32
    with gpu_sim(cfg, init, des) as g:
        J32, g32 = g.adjoint(adj)
    assert abs(J32 - J64) <= 1e-5 * abs(J64)
    for name in abi.DESIGN_NAMES:
        assert rel_l2(g32[name], g64[name]) <= 1e-4, (name, rel_l2(g32[name], g64[name]))


def test_fp64_adjoint_matches_gpu_finite_differences():
    """dJ/d(eps_inf, Delta-eps factor, chi factor) against central differences
    (h = 1e-4) of the GPU's FP64 objective at 8 seeded cells per map."""
    cfg = design_case(abi.MP_SOLVER_PLRC_NONLIN, abi.MP_CPML_ALL, n=(16, 12, 20), source=True)
    cfg.design_box[:] = (5, 12, 3, 10, 8, 14)
    des = design_maps(cfg, 22)
    init = clean_init(cfg, 23, smooth=True, scale=0.2)
    adj = abi.adjoint_config(abi.MP_OBJ_E2_BOX, (6, 11, 4, 9, 15, 18), 40, checkpoint_every=8)
    with gpu_sim(cfg, init, des) as g:
        J, grads = g.adjoint(adj)

    def objective(d):
        with gpu_sim(cfg, init, d) as s:
            return s.objective(adj)

    rng = np.random.default_rng(24)
    h = 1e-4
    for name in abi.DESIGN_NAMES:
        scale = np.max(np.abs(grads[name]))
        for _ in range(8):
            idx = tuple(int(rng.integers(0, n)) for n in grads[name].shape)
            dp = {k: v.copy() for k, v in des.items()}
            dm = {k: v.copy() for k, v in des.items()}
            dp[name][idx] += h
            dm[name][idx] -= h
            fd = (objective(dp) - objective(dm)) / (2 * h)
            assert abs(fd - grads[name][idx]) <= 1e-4 * max(abs(fd), 1e-3 * scale), (name, idx, fd, grads[name][idx])


def test_autograd_function_gives_the_adjoint_gradient():
    cfg = design_case(abi.MP_SOLVER_PLRC_NONLIN, abi.MP_CPML_Z, source=True)
    des = design_maps(cfg, 25)
    init = clean_init(cfg, 26, smooth=True, scale=0.2)
    adj = abi.adjoint_config(abi.MP_OBJ_SZ_PLANE, BOXES[abi.MP_OBJ_SZ_PLANE], 14)
    problem = adjoint.DesignProblem(cfg, init, adj)
    eps = torch.tensor(des["DesignEps"], dtype=torch.float64, device="cuda", requires_grad=True)
    chi = torch.tensor(des["DesignChiScale"], dtype=torch.float64, device="cuda", requires_grad=True)
    J = adjoint.design_objective(problem, eps, torch.tensor(des["DesignDepsScale"], dtype=torch.float64), chi)
    J.backward()
    with gpu_sim(cfg, init, des) as g:
        J_ref, g_ref = g.adjoint(adj)
    assert abs(J.item() - J_ref) <= 1e-14 * abs(J_ref)
    np.testing.assert_allclose(eps.grad.cpu().numpy(), g_ref["DesignEps"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(chi.grad.cpu().numpy(), g_ref["DesignChiScale"], rtol=1e-12, atol=0)
    # without gradients the forward runs mp_objective
    with torch.no_grad():
        J2 = adjoint.design_objective(problem, eps, torch.tensor(des["DesignDepsScale"]), chi)
    assert abs(J2.item() - J_ref) <= 1e-12 * abs(J_ref)
    problem.close()
