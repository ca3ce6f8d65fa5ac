"""CUDA FP64 form against the golden fixtures of the reference build, through
the C ABI: relative L2 <= 1e-12 per field (FP64 parity bar); the FP32 form
within 1e-5 on the cases and 1e-4 on the long workload runs."""
import os

import numpy as np
import pytest

from mpulse_b200 import abi, runtime
from tests.cases import rel_l2
from tests.golden_util import case_files, case_init, load, workload_files, workload_init

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", case_files(), ids=os.path.basename)
def test_gpu_fp64_reproduces_reference_case(path):
    d, cfg = load(path)
    init = case_init(d, cfg)
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.step(int(d["steps"]))
        for n in abi.FIELD_NAMES:
            assert rel_l2(g.download(n), d[n]) <= 1e-12, n
        # the plasma plug-ins' state, on the planes the E half updates
        for n in [n for n in abi.PLASMA_NAMES if n in d]:
            assert rel_l2(g.download(n)[1:-1], d[n][1:-1]) <= 1e-12, n


@pytest.mark.parametrize("precision,tol", [(abi.MP_FP64, 1e-12), (abi.MP_FP32, 1e-4)])
@pytest.mark.parametrize("path", workload_files(), ids=os.path.basename)
def test_gpu_reproduces_reference_workload(path, precision, tol):
    d, cfg = load(path)
    cfg.precision = precision
    init = workload_init(path, cfg)
    with runtime.Simulation(cfg) as g:
        if init:
            for n, v in init.items():
                g.upload(n, v)
        g.step(int(d["steps"]))
        j = int(d["slice_y"])
        full = {n: g.download(n) for n in abi.FIELD_NAMES}
    # error of each component relative to the whole field: in these
    # single-polarisation runs some components are rounding noise (1e-15)
    total = np.sqrt(sum(np.linalg.norm(d[n]) ** 2 for n in abi.FIELD_NAMES))
    for n in abi.FIELD_NAMES:
        err = np.linalg.norm(full[n][:, j, :] - d[n]) / total
        assert err <= tol, (n, err)
