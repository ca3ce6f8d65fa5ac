"""mp_objective_record + mp_adjoint_reverse (the adjoint in two calls, as an
autograd tape) against mp_adjoint on every kind of schedule: the whole history,
checkpoints every few steps, revolve under a device budget (several slots, one
slot), and the two-level schedule with segment checkpoints in host memory.  J,
the three gradients and the end state agree to the last bit; the record's
forward run leaves the state mp_objective leaves; every call that changes the
state releases the record."""
import numpy as np
import pytest

from mpulse_b200 import abi, runtime
from tests.test_adjoint_oracle import clean_init, design_case, design_maps
from tests.test_gpu_adjoint import BOXES, gpu_sim

pytestmark = pytest.mark.gpu

STEPS = 30


def schedules(cfg):
    """name -> (adjoint config, states of host checkpoint budget)."""
    box = BOXES[abi.MP_OBJ_E2_BOX]
    n = cfg.field_count()
    return {
        "whole_history": (abi.adjoint_config(abi.MP_OBJ_E2_BOX, box, STEPS), 0),
        "every_7": (abi.adjoint_config(abi.MP_OBJ_E2_BOX, box, STEPS, checkpoint_every=7), 0),
        "every_20": (abi.adjoint_config(abi.MP_OBJ_E2_BOX, box, STEPS, checkpoint_every=20), 0),
        "every_30": (abi.adjoint_config(abi.MP_OBJ_E2_BOX, box, STEPS, checkpoint_every=30), 0),
        "budget_3_slots": (abi.adjoint_config(abi.MP_OBJ_E2_BOX, box, STEPS, mem_budget=648.0 * n), 0),
        "budget_1_slot": (abi.adjoint_config(abi.MP_OBJ_E2_BOX, box, STEPS, mem_budget=516.0 * n), 0),
        "two_level": (abi.adjoint_config(abi.MP_OBJ_E2_BOX, box, STEPS, mem_budget=516.0 * n), 12),
    }


def setup(cfg, init, des, host_states):
    g = gpu_sim(cfg, init, des)
    if host_states:
        g.set_host_checkpoint_budget(host_states * len(g.save_state()))
    return g


@pytest.mark.parametrize("precision", [abi.MP_FP64, abi.MP_FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("schedule", ["whole_history", "every_7", "every_20", "every_30", "budget_3_slots",
                                      "budget_1_slot", "two_level"])
def test_record_and_reverse_equal_adjoint(schedule, precision):
    cfg = design_case(abi.MP_SOLVER_PLRC_NONLIN, abi.MP_CPML_Z, source=True)
    cfg.precision = precision
    des = design_maps(cfg, 31)
    init = clean_init(cfg, 32, smooth=True, scale=0.2)
    adj, host_states = schedules(cfg)[schedule]
    with setup(cfg, init, des, host_states) as g:
        J0, g0 = g.adjoint(adj)
        end0 = g.save_state()
    with gpu_sim(cfg, init, des) as g:
        Jf = g.objective(adj)
        endf = g.save_state()
    with setup(cfg, init, des, host_states) as g:
        Jr = g.objective_record(adj)
        assert g.time == STEPS
        assert g.save_state() == endf  # the record's forward run is mp_objective's
        J1, g1 = g.adjoint_reverse()
        assert g.time == STEPS
        end1 = g.save_state()
    assert Jr == Jf == J0 == J1
    assert end1 == end0 == endf
    for name in abi.DESIGN_NAMES:
        assert np.array_equal(g1[name], g0[name]), name
    assert np.any(g1["DesignEps"])


@pytest.mark.parametrize("every,host_states", [(7, 0), (0, 12)], ids=["every_7", "two_level"])
def test_record_and_reverse_sz_plane(every, host_states):
    """The Sz-plane objective, whose history also keeps Bx and By on the plane,
    in a linear medium (E history stored only at the design cells and on the
    plane)."""
    cfg = design_case(abi.MP_SOLVER_PLRC_LIN, abi.MP_CPML_ALL, source=True)
    des = design_maps(cfg, 41)
    init = clean_init(cfg, 42, smooth=True, scale=0.2)
    box = BOXES[abi.MP_OBJ_SZ_PLANE]
    if every:
        adj = abi.adjoint_config(abi.MP_OBJ_SZ_PLANE, box, STEPS, checkpoint_every=every)
    else:
        adj = abi.adjoint_config(abi.MP_OBJ_SZ_PLANE, box, STEPS, mem_budget=516.0 * cfg.field_count())
    with setup(cfg, init, des, host_states) as g:
        J0, g0 = g.adjoint(adj)
    with setup(cfg, init, des, host_states) as g:
        Jr = g.objective_record(adj)
        J1, g1 = g.adjoint_reverse()
    assert Jr == J0 == J1
    for name in abi.DESIGN_NAMES:
        assert np.array_equal(g1[name], g0[name]), name
    assert np.any(g1["DesignEps"])


def test_reverse_twice_and_without_record():
    cfg = design_case(abi.MP_SOLVER_PLRC_LIN, abi.MP_CPML_Z, source=True)
    des = design_maps(cfg, 33)
    init = clean_init(cfg, 34, smooth=True, scale=0.2)
    adj = abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], 12, checkpoint_every=5)
    with gpu_sim(cfg, init, des) as g:
        with pytest.raises(runtime.MPulseError):
            g.adjoint_reverse()
        g.objective_record(adj)
        g.adjoint_reverse()
        with pytest.raises(runtime.MPulseError):
            g.adjoint_reverse()  # the record is used up
        # a second record replaces the first; releasing twice is harmless
        g.objective_record(adj)
        g.objective_record(adj)
        g.release_record()
        g.release_record()
        with pytest.raises(runtime.MPulseError):
            g.adjoint_reverse()


MUTATORS = {
    "step": lambda g, s: g.step(1),
    "kernel_times": lambda g, s: g.kernel_times(1),
    "upload_field": lambda g, s: g.upload("Ex", np.zeros(g.cfg.field_count())),
    "upload_design": lambda g, s: g.upload_design("DesignEps", g.download_design("DesignEps")),
    "set_time": lambda g, s: setattr(g, "time", g.time),
    "load_state": lambda g, s: g.load_state(s),
    "objective": lambda g, s: g.objective(abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], 2)),
    "host_budget": lambda g, s: g.set_host_checkpoint_budget(0),
    "set_stream": lambda g, s: g.set_stream(None),
    "release": lambda g, s: g.release_record(),
}


@pytest.mark.parametrize("mutator", sorted(MUTATORS))
def test_state_changes_release_the_record(mutator):
    cfg = design_case(abi.MP_SOLVER_PLRC_LIN, abi.MP_CPML_Z, source=True)
    des = design_maps(cfg, 35)
    init = clean_init(cfg, 36, smooth=True, scale=0.2)
    adj = abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], 12, checkpoint_every=5)
    with gpu_sim(cfg, init, des) as g:
        g.objective_record(adj)
        saved = g.save_state()
        MUTATORS[mutator](g, saved)
        with pytest.raises(runtime.MPulseError, match="no recorded run"):
            g.adjoint_reverse()


def test_reads_keep_the_record():
    """Downloads, the energy and saving the state read the context and keep
    the record."""
    cfg = design_case(abi.MP_SOLVER_PLRC_LIN, abi.MP_CPML_Z, source=True)
    des = design_maps(cfg, 37)
    init = clean_init(cfg, 38, smooth=True, scale=0.2)
    adj = abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], 12, checkpoint_every=5)
    with gpu_sim(cfg, init, des) as g:
        J0, g0 = g.adjoint(adj)
    with gpu_sim(cfg, init, des) as g:
        g.objective_record(adj)
        g.download("Ex")
        g.download_design("DesignEps")
        g.field_energy()
        g.save_state()
        J1, g1 = g.adjoint_reverse()
    assert J1 == J0
    for name in abi.DESIGN_NAMES:
        assert np.array_equal(g1[name], g0[name]), name


def test_autograd_backward_after_another_evaluation():
    """Two evaluations of one problem before backward: the first one's record
    was released by the second, so its backward runs mp_adjoint from the
    initial state; both gradients equal mp_adjoint's."""
    import torch
    from mpulse_b200 import adjoint

    cfg = design_case(abi.MP_SOLVER_PLRC_NONLIN, abi.MP_CPML_Z, source=True)
    des = design_maps(cfg, 39)
    init = clean_init(cfg, 40, smooth=True, scale=0.2)
    adj = abi.adjoint_config(abi.MP_OBJ_E2_BOX, BOXES[abi.MP_OBJ_E2_BOX], 14, checkpoint_every=5)
    problem = adjoint.DesignProblem(cfg, init, adj)
    eps1 = torch.tensor(des["DesignEps"], dtype=torch.float64, requires_grad=True)
    eps2 = torch.tensor(des["DesignEps"] * 1.01, dtype=torch.float64, requires_grad=True)
    J1 = adjoint.design_objective(problem, eps1)
    J2 = adjoint.design_objective(problem, eps2)
    (J1 + J2).backward()
    problem.close()
    for eps, t in ((eps1, des["DesignEps"]), (eps2, des["DesignEps"] * 1.01)):
        # the other maps keep their defaults, as in the evaluations above
        with gpu_sim(cfg, init, {"DesignEps": t}) as g:
            _, ref = g.adjoint(adj)
        assert np.array_equal(eps.grad.numpy(), ref["DesignEps"])
