"""Known answer about the reference scheme itself, pinned on the oracle (which
reproduces the reference bit for bit): MPulse's PLRC update with eps_inf = 1 and
the 68.4 nm Sellmeier pole, at dx = 40 nm, amplifies grid-scale perturbations at
dt = 0.5 dx / c and is stable at dt = 0.45 dx / c, the value the workloads with
that medium use.  If the reference build is present the same growth is checked
on it directly."""
import os

import numpy as np
import pytest

from mpulse_b200 import abi, configs
from oracle import pyoracle
from tests.cases import make_case, random_fields


def _cfg(courant, eps=1.0):
    cfg = make_case("lin_all_wave_periodic", abi.MP_FP64)
    cfg.n_sources = 0
    cfg.cpml = abi.MP_CPML_NONE
    cfg.eps = eps
    cfg.dt = courant * cfg.dx
    return cfg


def _growth(cfg, steps=100):
    init = random_fields(cfg, seed=5, scale=1e-3)
    o = pyoracle.OracleSim(cfg)
    for n, v in init.items():
        o.upload(n, v)
    n0 = np.sqrt(sum(np.sum(v ** 2) for v in init.values()))
    o.step(steps)
    return np.sqrt(sum(np.sum(o.download(n) ** 2) for n in abi.FIELD_NAMES)) / n0


def test_plrc_unstable_at_half_courant_with_eps_inf_one():
    assert _growth(_cfg(0.5)) > 1e6


def test_plrc_stable_at_medium_courant():
    assert _growth(_cfg(configs.MEDIUM_COURANT)) < 2.0
    assert _growth(_cfg(0.5, eps=1.2)) < 2.0


@pytest.mark.skipif(not os.path.exists(pyoracle.REF_BIN), reason="reference build not present")
def test_reference_build_shows_the_same_growth():
    cfg = _cfg(0.5)
    init = random_fields(cfg, seed=5, scale=1e-3)
    ref, _ = pyoracle.run_reference(cfg, 60, init)
    o = pyoracle.OracleSim(cfg)
    for n, v in init.items():
        o.upload(n, v)
    o.step(60)
    for n in abi.FIELD_NAMES:
        np.testing.assert_array_equal(o.download(n), ref[n])
    assert max(np.abs(ref[n]).max() for n in ref) > 1e2
