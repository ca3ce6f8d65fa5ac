"""torch.autograd.Function over mp_adjoint: the objective of a run as a
differentiable function of the design maps.

    problem = DesignProblem(cfg, init_fields, adj)        # cfg has a design_box
    eps = torch.full(abi.design_shape(cfg), 2.0, dtype=torch.float64, requires_grad=True)
    J = design_objective(problem, eps)                    # Delta-eps / chi factors optional
    J.backward()                                          # eps.grad = dJ/d eps_inf per cell

Every evaluation starts from the problem's initial state (fields, PLRC and CPML
state zero, time `start_time`).  When any input requires a gradient the
forward call runs mp_objective_record (the forward run keeping mp_adjoint's
checkpoints) and backward runs mp_adjoint_reverse (the reverse pass) on the
same simulation; otherwise forward runs mp_objective.  If another evaluation
of the problem has replaced the simulation before backward, backward runs
mp_adjoint from the initial state with the maps of its own forward call (the
same gradient).
The maps travel as FP64 host arrays through the C ABI; the result has the
dtype and device of the first map.
"""
from __future__ import annotations

import torch

from . import abi, runtime


class DesignProblem:
    """A configuration, its initial fields and the objective of mp_adjoint."""

    def __init__(self, cfg: abi.Config, init_fields: dict | None, adj: abi.AdjointConfig, start_time: int = 0):
        if abi.design_shape(cfg) is None:
            raise ValueError("the configuration has no design box")
        self.cfg = cfg
        self.init = init_fields or {}
        self.adj = adj
        self.start_time = start_time
        self.sim = None

    def reset(self, maps: dict):
        """A fresh simulation (all state zero) with the initial fields, the start
        time and the given design maps."""
        self.close()
        sim = self.sim = runtime.Simulation(self.cfg)
        for name, arr in self.init.items():
            sim.upload(name, arr)
        sim.time = self.start_time
        for name, arr in maps.items():
            sim.upload_design(name, arr)
        return sim

    def close(self):
        if self.sim is not None:
            self.sim.close()
            self.sim = None


class DesignObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, problem: DesignProblem, eps, dscale, chiscale):
        shape = abi.design_shape(problem.cfg)
        maps = {}
        for name, t in zip(abi.DESIGN_NAMES, (eps, dscale, chiscale)):
            if t is not None:
                maps[name] = t.detach().to("cpu", torch.float64).numpy().reshape(shape)
        sim = problem.reset(maps)
        ref = eps if eps is not None else (dscale if dscale is not None else chiscale)
        ctx.problem, ctx.maps, ctx.sim = problem, maps, sim
        ctx.device, ctx.dtype = ref.device, ref.dtype
        if any(ctx.needs_input_grad[1:]):
            J = sim.objective_record(problem.adj)
        else:
            J = sim.objective(problem.adj)
        return torch.tensor(J, dtype=ref.dtype, device=ref.device)

    @staticmethod
    def backward(ctx, gJ):
        problem = ctx.problem
        grads = None
        if problem.sim is ctx.sim:
            try:
                _, grads = ctx.sim.adjoint_reverse()
            except runtime.MPulseError:
                grads = None  # the record was released: run the whole adjoint below
        if grads is None:
            _, grads = problem.reset(ctx.maps).adjoint(problem.adj)
        ctx.sim = None
        out = [None]
        for k, name in enumerate(abi.DESIGN_NAMES):
            g = torch.from_numpy(grads[name]).to(ctx.device, ctx.dtype)
            out.append(gJ * g if ctx.needs_input_grad[1 + k] else None)
        return tuple(out)


def design_objective(problem: DesignProblem, eps=None, dscale=None, chiscale=None):
    """J(eps_inf, Delta-eps factor, chi factor) over the problem's design box;
    a map left None keeps the values set in the simulation (defaults eps, 1, 1)."""
    if eps is None and dscale is None and chiscale is None:
        raise ValueError("give at least one design map")
    return DesignObjective.apply(problem, eps, dscale, chiscale)
