"""The oracle against the golden fixtures made by running the reference build
(tests/golden/make_golden.py): bit-for-bit on the parity cases, relative L2
<= 1e-13 on the workload slices and on the cases whose source goes through
transcendental code of the oracle's own (the short pulse's Faddeeva function;
the gauss beam's DFTs, which the reference build takes from the direct-DFT
stand-in for FFTW in oracle/refshim/fftw_shim.cpp)."""
import os

import numpy as np
import pytest

from mpulse_b200 import abi
from oracle import pyoracle
from tests.cases import rel_l2
from tests.golden_util import case_files, case_init, load, workload_files, workload_init


@pytest.mark.parametrize("path", case_files(), ids=os.path.basename)
def test_oracle_reproduces_reference_case(path):
    d, cfg = load(path)
    init = case_init(d, cfg)
    o = pyoracle.OracleSim(cfg)
    for n, v in init.items():
        o.upload(n, v)
    assert o.step(int(d["steps"])) == abi.MP_OK
    # the fields, and the plasma plug-ins' density and current where the case has them
    for n in [n for n in abi.FIELD_NAMES + abi.PLASMA_NAMES if n in d]:
        got = o.download(n)
        if cfg.n_sources and cfg.sources[0].kind in (abi.MP_SOURCE_SHORT_PULSE, abi.MP_SOURCE_GAUSS_BEAM):
            assert rel_l2(got, d[n]) <= 1e-13, n
        else:
            np.testing.assert_array_equal(got, d[n], err_msg=n)


@pytest.mark.parametrize("path", workload_files(), ids=os.path.basename)
def test_oracle_reproduces_reference_workload(path):
    d, cfg = load(path)
    init = workload_init(path, cfg)
    o = pyoracle.OracleSim(cfg)
    if init:
        for n, v in init.items():
            o.upload(n, v)
    assert o.step(int(d["steps"])) == abi.MP_OK
    j = int(d["slice_y"])
    full = {n: o.download(n) for n in abi.FIELD_NAMES}
    total = np.sqrt(sum(np.linalg.norm(d[n]) ** 2 for n in abi.FIELD_NAMES))
    for n in abi.FIELD_NAMES:
        assert np.linalg.norm(full[n][:, j, :] - d[n]) <= 1e-13 * total, n
    energy = sum(np.sum(full[n][1:-1] ** 2) for n in abi.FIELD_NAMES)
    assert abs(energy - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))


def test_oracle_energy_matches_reference_diagnostic():
    """mpo_field_energy restates FieldEnergyDiag::calculate; the workload
    fixtures hold the reference's sum(E^2 + B^2) over the interior."""
    for path in workload_files():
        d, cfg = load(path)
        init = workload_init(path, cfg)
        o = pyoracle.OracleSim(cfg)
        if init:
            for n, v in init.items():
                o.upload(n, v)
        o.step(int(d["steps"]))
        e = o.field_energy() / (cfg.dx * cfg.dy * cfg.dz)
        assert abs(e - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))
