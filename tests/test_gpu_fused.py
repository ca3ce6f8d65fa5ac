"""The fused step form (staging FUSED: both half steps of a tile of columns in
one z-march, the tiles' edge cells in a second kernel) against the two
half-step kernels (staging GLOBAL): the whole device state after the same
steps (fields, PLRC accumulators, CPML psi, time: mp_save_state) is identical
byte for byte, in FP32 and FP64 (within rounding where GLOBAL's B half is the
vector kernel).  The cases cover every solver, boundary,
CPML kind and source kind of the parity suite, grids whose sizes are not
multiples of the 32 x 8 tile, grids smaller than one tile, and runs long
enough to cross the z-chunks' top planes and the source batches."""
import zlib

import pytest

from mpulse_b200 import abi, runtime
from tests.cases import CASES, make_case, random_fields, rel_l2

pytestmark = pytest.mark.gpu
STEPS = 30

# the fused form leaves out design regions and the plasma plug-ins
FUSABLE = sorted(c for c in CASES if "plasma" not in c)


def state_after(cfg, init, staging, steps):
    cfg.staging = staging
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.step(steps)
        return g.save_state()


def fields_after(cfg, init, staging, steps):
    cfg.staging = staging
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.step(steps)
        return {n: g.download(n) for n in abi.FIELD_NAMES}


def assert_same(cfg, seed, steps=STEPS):
    """Byte for byte where GLOBAL runs the scalar B half (b_cell, as the fused
    form does); where nx is a multiple of 64 GLOBAL runs the vector B half,
    whose own copy of the arithmetic may round a multiply-add differently, so
    there the fields agree within rounding."""
    init = random_fields(cfg, seed=seed)
    if cfg.nx % 64 != 0:
        split = state_after(cfg, init, abi.MP_STAGING_GLOBAL, steps)
        fused = state_after(cfg, init, abi.MP_STAGING_FUSED, steps)
        assert len(split) == len(fused)
        assert split == fused
    else:
        tol = 1e-14 if cfg.precision == abi.MP_FP64 else 1e-6
        split = fields_after(cfg, init, abi.MP_STAGING_GLOBAL, steps)
        fused = fields_after(cfg, init, abi.MP_STAGING_FUSED, steps)
        for n in abi.FIELD_NAMES:
            assert rel_l2(fused[n], split[n]) <= tol, n


@pytest.mark.parametrize("prec", [abi.MP_FP32, abi.MP_FP64], ids=["fp32", "fp64"])
@pytest.mark.parametrize("case", FUSABLE)
def test_fused_state_equals_split(case, prec):
    assert_same(make_case(case, prec), zlib.crc32(case.encode()) % 1000)


@pytest.mark.parametrize("shape", [(33, 9, 17), (31, 7, 9), (5, 3, 6), (64, 16, 40), (40, 24, 3)])
@pytest.mark.parametrize("case", ["nonlin_all_short", "plain_periodic", "nl_xy", "lin_all_wave_periodic"])
def test_fused_odd_and_small_grids(case, shape):
    cfg = make_case(case, abi.MP_FP64)
    cfg.nx, cfg.ny, cfg.nz = shape
    cfg.medium_z0, cfg.medium_z1 = 0, cfg.nz + 1
    cfg.cpml_d = min(cfg.cpml_d, max(1, min(shape) // 2 - 1))
    for q in range(cfg.n_sources):
        cfg.sources[q].distance = min(cfg.sources[q].distance, cfg.nz - 1)
    try:
        runtime.Simulation(cfg).close()
    except runtime.MPulseError as e:
        pytest.skip(f"configuration rejected: {e}")
    assert_same(cfg, sum(shape), steps=20)


def test_fused_long_run_fp32():
    """200 steps of the short-pulse case: the source batches of 64 steps and
    the z-chunks' top planes in every step."""
    cfg = make_case("nonlin_all_short", abi.MP_FP32)
    assert_same(cfg, 7, steps=200)


def test_fused_rejects_plasma_and_design():
    cfg = make_case("plasma_nonlin_all_short", abi.MP_FP32)
    cfg.staging = abi.MP_STAGING_FUSED
    with pytest.raises(runtime.MPulseError):
        runtime.Simulation(cfg)
