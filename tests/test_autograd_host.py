"""The host logic of the autograd wrapper (mpulse_b200/adjoint.py) with a fake
simulation in place of the library: which entry points forward and backward
call, and the way back to mp_adjoint when the record of a forward call was
released before its backward ran.  No GPU."""
import numpy as np
import pytest
import torch

from mpulse_b200 import abi, adjoint, runtime

SHAPE = (2, 3, 4)


class FakeSim:
    """Stands in for runtime.Simulation: J and the gradients are functions of
    the uploaded DesignEps map, so every call's inputs can be checked."""

    log = []

    def __init__(self, cfg):
        self.maps = {}
        self.recorded = False
        self.closed = False

    def upload(self, name, arr):
        pass

    def upload_design(self, name, arr):
        self.maps[name] = np.array(arr, dtype=np.float64)

    @property
    def time(self):
        return 0

    @time.setter
    def time(self, t):
        pass

    def _J(self):
        return float(np.sum(self.maps["DesignEps"] ** 2))

    def _grads(self):
        e = self.maps["DesignEps"]
        return {"DesignEps": 2 * e, "DesignDepsScale": np.zeros_like(e), "DesignChiScale": np.ones_like(e)}

    def objective(self, adj):
        FakeSim.log.append("objective")
        return self._J()

    def objective_record(self, adj):
        FakeSim.log.append("record")
        self.recorded = True
        return self._J()

    def adjoint_reverse(self):
        FakeSim.log.append("reverse")
        if not self.recorded or self.closed:
            raise runtime.MPulseError(abi.MP_ERR_INVALID, "no recorded run")
        self.recorded = False
        return self._J(), self._grads()

    def adjoint(self, adj):
        FakeSim.log.append("adjoint")
        return self._J(), self._grads()

    def close(self):
        self.closed = True


@pytest.fixture
def problem(monkeypatch):
    monkeypatch.setattr(runtime, "Simulation", FakeSim)
    monkeypatch.setattr(abi, "design_shape", lambda cfg: SHAPE)
    FakeSim.log = []
    adj = abi.adjoint_config(abi.MP_OBJ_E2_BOX, (1, 1, 1, 1, 1, 1), 4)
    p = adjoint.DesignProblem(abi.default_config(), {}, adj)
    yield p
    p.close()


def test_forward_records_and_backward_reverses(problem):
    e = torch.rand(SHAPE, dtype=torch.float64, requires_grad=True)
    J = adjoint.design_objective(problem, e)
    assert FakeSim.log == ["record"]
    J.backward()
    assert FakeSim.log == ["record", "reverse"]
    assert torch.allclose(e.grad, 2 * e.detach())
    assert J.item() == pytest.approx(float((e.detach() ** 2).sum()))


def test_backward_after_another_evaluation_runs_the_whole_adjoint(problem):
    e1 = torch.rand(SHAPE, dtype=torch.float64, requires_grad=True)
    e2 = torch.rand(SHAPE, dtype=torch.float64, requires_grad=True)
    J1 = adjoint.design_objective(problem, e1)
    J2 = adjoint.design_objective(problem, e2)
    J1.backward()  # the problem's simulation is now J2's: J1's record is gone
    assert FakeSim.log == ["record", "record", "adjoint"]
    assert torch.allclose(e1.grad, 2 * e1.detach())  # the gradient at J1's own maps
    J2.backward()  # J1's backward replaced the simulation too
    assert FakeSim.log[-1] == "adjoint"
    assert torch.allclose(e2.grad, 2 * e2.detach())


def test_released_record_falls_back(problem):
    e = torch.rand(SHAPE, dtype=torch.float64, requires_grad=True)
    J = adjoint.design_objective(problem, e)
    problem.sim.recorded = False  # as after a call that releases the record
    J.backward()
    assert FakeSim.log == ["record", "reverse", "adjoint"]
    assert torch.allclose(e.grad, 2 * e.detach())


def test_no_gradient_runs_the_objective(problem):
    e = torch.rand(SHAPE, dtype=torch.float64)
    J = adjoint.design_objective(problem, e)
    assert FakeSim.log == ["objective"]
    assert J.item() == pytest.approx(float((e ** 2).sum()))


def test_gradients_only_for_inputs_that_need_them(problem):
    e = torch.rand(SHAPE, dtype=torch.float64, requires_grad=True)
    chi = torch.rand(SHAPE, dtype=torch.float64, requires_grad=True)
    d = torch.rand(SHAPE, dtype=torch.float64)  # no gradient wanted
    J = adjoint.design_objective(problem, e, d, chi)
    J.backward()
    assert torch.allclose(chi.grad, torch.ones(SHAPE, dtype=torch.float64))
    assert d.grad is None
