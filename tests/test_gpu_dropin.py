"""The drop-in end to end: MPulse's own driver (setup-file parser, Process
time loop, FieldSimulation, Storage, boundary objects) built from its sources,
once with its CPU solver and once with the B200 FieldSolver plug-in
(mpulse_b200/host/fdtd_gpu.cpp) registered as fdtd-gpu-*, on the same setup
file and initial fields.  FP64: relative L2 <= 1e-12 per field."""
import os

import pytest

from mpulse_b200 import abi
from oracle import pyoracle
from tests.cases import make_case, random_fields, rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(pyoracle.REF_BIN) and os.path.exists(pyoracle.REF_BIN_GPU)),
                                 reason="reference builds not present (make -C oracle ref gpuref)")]

GPU_NAMES = {
    abi.MP_SOLVER_PLAIN: "fdtd-gpu-plain",
    abi.MP_SOLVER_NL: "fdtd-gpu-nl",
    abi.MP_SOLVER_PLRC_LIN: "fdtd-gpu-plrc-lin",
    abi.MP_SOLVER_PLRC_NONLIN: "fdtd-gpu-plrc-nonlin",
}


@pytest.mark.parametrize("case", ["nonlin_all_short", "lin_split_cpmlz_gauss", "plain_xy", "nl_periodic",
                                  "nonlin_three_poles", "nonlin_all_gauss_beam_blocks", "plasma_nonlin_all_short"])
def test_mpulse_driver_with_gpu_solver(case):
    cfg = make_case(case, abi.MP_FP64)
    init = random_fields(cfg, seed=21)
    plasma = abi.PLASMA_NAMES if (cfg.plasma or cfg.plasma_current) else ()
    names = abi.FIELD_NAMES + plasma
    cpu, _ = pyoracle.run_reference(cfg, 20, init, names=names)
    gpu, _ = pyoracle.run_reference(cfg, 20, init, names=names, binary=pyoracle.REF_BIN_GPU,
                                    solver_name=GPU_NAMES[cfg.solver], extra="sync_interval 1")
    for n in abi.FIELD_NAMES:
        assert rel_l2(gpu[n], cpu[n]) <= 1e-12, (n, rel_l2(gpu[n], cpu[n]))
    for n in plasma:  # the plug-in keeps the plasma state on the planes the E half updates
        assert rel_l2(gpu[n][1:-1], cpu[n][1:-1]) <= 1e-12, (n, rel_l2(gpu[n][1:-1], cpu[n][1:-1]))


def test_sync_interval_keeps_device_state():
    """With sync_interval 0 the Storage grids are never refreshed, but the
    device state advances; with 5 they are refreshed every 5 steps."""
    cfg = make_case("lin_split_cpmlz_gauss", abi.MP_FP64)
    init = random_fields(cfg, seed=22)
    cpu, _ = pyoracle.run_reference(cfg, 10, init)
    gpu, _ = pyoracle.run_reference(cfg, 10, init, binary=pyoracle.REF_BIN_GPU, solver_name="fdtd-gpu-plrc-lin",
                                    extra="sync_interval 5")
    for n in abi.FIELD_NAMES:
        assert rel_l2(gpu[n], cpu[n]) <= 1e-12
