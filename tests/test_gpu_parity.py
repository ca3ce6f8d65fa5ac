"""CUDA path vs the FP64 CPU oracle on the same seeded inputs, through the C ABI.

FP64 form: relative L2 error <= 1e-12 per field (the oracle reproduces the
reference bit for bit, see test_oracle_reference.py).  FP32 form: relative L2
error <= 1e-5 against the FP64 oracle (the precision target of the FP32 form).
"""
import zlib

import numpy as np
import pytest

from mpulse_b200 import abi, runtime
from oracle import pyoracle
from tests.cases import CASES, make_case, random_fields, rel_l2

TOL_FP64 = 1e-12
TOL_FP32 = 1e-5
STEPS = 25

pytestmark = pytest.mark.gpu


def run_pair(cfg, init, steps, names=abi.FIELD_NAMES):
    o = pyoracle.OracleSim(cfg)
    for n, v in init.items():
        o.upload(n, v)
    rc = o.step(steps)
    assert rc == abi.MP_OK
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.step(steps)
        assert g.time == steps
        got = {n: g.download(n) for n in names}
    want = {n: o.download(n) for n in names}
    return got, want


def psi_names(cfg):
    if cfg.solver not in (abi.MP_SOLVER_PLRC_LIN, abi.MP_SOLVER_PLRC_NONLIN):
        return ()
    return tuple(f"Psi{ri}{n + 1}{c}" for ri in "RI" for n in range(3) if cfg.poles[n].eps != 0 for c in "xyz")


def plasma_names(cfg):
    """The plasma plug-ins' state; the device keeps it on the planes 1..nz the
    E half updates, so it is compared there."""
    return abi.PLASMA_NAMES if (cfg.plasma or cfg.plasma_current) else ()


def interior(name, a):
    return a[1:-1] if name in abi.PLASMA_NAMES else a


@pytest.mark.parametrize("case", sorted(CASES))
def test_fp64_matches_oracle(case):
    cfg = make_case(case, abi.MP_FP64)
    init = random_fields(cfg, seed=zlib.crc32(case.encode()) % 1000)
    names = abi.FIELD_NAMES + psi_names(cfg) + plasma_names(cfg)
    got, want = run_pair(cfg, init, STEPS, names)
    for n in names:
        err = rel_l2(interior(n, got[n]), interior(n, want[n]))
        assert err <= TOL_FP64, f"{case} {n}: rel-L2 {err:.3e}"


@pytest.mark.parametrize("case", sorted(CASES))
def test_fp32_matches_oracle(case):
    cfg32 = make_case(case, abi.MP_FP32)
    cfg64 = make_case(case, abi.MP_FP64)
    init = random_fields(cfg64, seed=7 + zlib.crc32(case.encode()) % 1000, smooth=True)
    o = pyoracle.OracleSim(cfg64)
    for n, v in init.items():
        o.upload(n, v)
    o.step(STEPS)
    with runtime.Simulation(cfg32) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.step(STEPS)
        for n in abi.FIELD_NAMES + plasma_names(cfg64):
            err = rel_l2(interior(n, g.download(n)), interior(n, o.download(n)))
            assert err <= TOL_FP32, f"{case} {n}: rel-L2 {err:.3e}"


def test_upload_download_roundtrip_and_ghosts():
    cfg = make_case("plain_periodic", abi.MP_FP64)
    init = random_fields(cfg, seed=3)
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        for n, v in init.items():
            np.testing.assert_array_equal(g.download(n), v)


def test_newton_cap_reports_error_without_fault():
    cfg = make_case("nonlin_one_pole_periodic", abi.MP_FP64)
    cfg.chi = 50.0
    cfg.newton_max_iter = 1
    init = random_fields(cfg, seed=5, scale=2.0)
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        with pytest.raises(runtime.MPulseError) as ei:
            g.step(2)
        assert ei.value.code == abi.MP_ERR_NEWTON
        # the context stays usable
        cfg2 = make_case("nonlin_one_pole_periodic", abi.MP_FP64)
        g2 = runtime.Simulation(cfg2)
        g2.step(1)
        g2.close()


def test_time_counter_and_sources_follow_process_time():
    """Setting the time moves the injected pulse exactly like Process::time."""
    cfg = make_case("lin_split_cpmlz_gauss", abi.MP_FP64)
    o = pyoracle.OracleSim(cfg)
    o.time = 40
    o.step(10)
    with runtime.Simulation(cfg) as g:
        g.time = 40
        g.step(10)
        assert g.time == 50
        for n in abi.FIELD_NAMES:
            assert rel_l2(g.download(n), o.download(n)) <= TOL_FP64


@pytest.mark.parametrize("precision,tol", [(abi.MP_FP64, TOL_FP64), (abi.MP_FP32, TOL_FP32)])
def test_sources_computed_ahead_follow_single_steps_and_time_jumps(precision, tol):
    """The injection planes are computed a batch ahead on a second stream, in
    buffers keyed by the steps they hold.  Single steps across a batch
    boundary (the batch is 64 steps here), a jump back in time and a jump
    forward past both buffers give the oracle's fields."""
    cfg = make_case("lin_split_cpmlz_gauss", precision)
    cfg64 = make_case("lin_split_cpmlz_gauss", abi.MP_FP64)
    init = random_fields(cfg64, seed=17, smooth=True, scale=0.05)
    o = pyoracle.OracleSim(cfg64)
    for n, v in init.items():
        o.upload(n, v)
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        for _ in range(70):  # one step per call, across the first batch boundary
            g.step(1)
        assert o.step(70) == abi.MP_OK
        for n in abi.FIELD_NAMES:
            assert rel_l2(g.download(n), o.download(n)) <= tol, n
        g.time = 30  # back into the first batch
        o.time = 30
        g.step(50)
        assert o.step(50) == abi.MP_OK
        for n in abi.FIELD_NAMES:
            assert rel_l2(g.download(n), o.download(n)) <= tol, n
        g.time = 400  # beyond both buffers
        o.time = 400
        g.step(5)
        assert o.step(5) == abi.MP_OK
        for n in abi.FIELD_NAMES:
            assert rel_l2(g.download(n), o.download(n)) <= tol, n


@pytest.mark.parametrize("start,steps", [(21, 30), (0, 60), (45, 8)])
def test_gauss_beam_blocks_follow_process_time(start, steps):
    """gauss_inject with Nt = 16 and t_size = 40: blocks start at 0, 16, 32 and
    the source is off from 48 on.  Entering mid-block through mp_set_time
    computes the block holding the time; stepping on crosses into the next block
    and past the switch-off like the oracle."""
    cfg = make_case("nonlin_all_gauss_beam_blocks", abi.MP_FP64)
    init = random_fields(cfg, seed=11 + start, scale=0.05)
    o = pyoracle.OracleSim(cfg)
    for n, v in init.items():
        o.upload(n, v)
    o.time = start
    assert o.step(steps) == abi.MP_OK
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.time = start
        g.step(steps)
        for n in abi.FIELD_NAMES:
            err = rel_l2(g.download(n), o.download(n))
            assert err <= TOL_FP64, f"{n}: rel-L2 {err:.3e}"


@pytest.mark.parametrize("precision,tol", [(abi.MP_FP64, 1e-13), (abi.MP_FP32, 1e-5)])
def test_field_energy_matches_oracle(precision, tol):
    """mp_field_energy against the oracle's restatement of
    FieldEnergyDiag::calculate (fielddiag.cpp:255-286)."""
    cfg = make_case("nonlin_odd_sizes", precision)
    cfg64 = make_case("nonlin_odd_sizes", abi.MP_FP64)
    init = random_fields(cfg64, seed=31, smooth=True)
    o = pyoracle.OracleSim(cfg64)
    for n, v in init.items():
        o.upload(n, v)
    o.step(7)
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.step(7)
        e = g.field_energy()
    ref = o.field_energy()
    assert abs(e - ref) <= tol * abs(ref)


@pytest.mark.parametrize("precision,tol", [(abi.MP_FP64, 1e-14), (abi.MP_FP32, 1e-6)])
@pytest.mark.parametrize("case", sorted(c for c in CASES if c.startswith("tma_")))
def test_tma_and_global_kernels_agree(case, precision, tol):
    """The TMA-staged kernels and the global-load kernels (whose B half loads
    16-byte vectors along x) run the same cell arithmetic on the same values;
    they differ only where the compiler fuses a multiply and an add in one
    kernel and not in the other (a last-bit rounding difference)."""
    out = []
    for staging in (abi.MP_STAGING_TMA, abi.MP_STAGING_GLOBAL):
        cfg = make_case(case, precision)
        cfg.staging = staging
        init = random_fields(cfg, seed=51)
        with runtime.Simulation(cfg) as g:
            for n, v in init.items():
                g.upload(n, v)
            g.step(9)
            out.append({n: g.download(n) for n in abi.FIELD_NAMES})
    for n in abi.FIELD_NAMES:
        assert rel_l2(out[0][n], out[1][n]) <= tol, n


@pytest.mark.parametrize("case", ["tma_nonlin_all_short", "tma_lin_periodic_three_poles"])
def test_tma_kernels_match_oracle(case):
    cfg = make_case(case, abi.MP_FP64)
    cfg.staging = abi.MP_STAGING_TMA
    init = random_fields(cfg, seed=52)
    got, want = run_pair(cfg, init, STEPS)
    for n in abi.FIELD_NAMES:
        assert rel_l2(got[n], want[n]) <= TOL_FP64, n


@pytest.mark.parametrize("case", ["nonlin_all_short", "lin_cpmlz_gauss_beam", "nonlin_three_poles"])
def test_save_and_load_state_resumes_bit_for_bit(case):
    """mp_save_state / mp_load_state: a run resumed from a saved state, in the
    same context or a new one, continues exactly like the uninterrupted run."""
    cfg = make_case(case, abi.MP_FP32)
    init = random_fields(cfg, seed=5, smooth=True)
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.step(7)
        snap = g.save_state()
        g.step(9)
        want = {n: g.download(n) for n in abi.FIELD_NAMES}
        g.step(3)
        g.load_state(snap)
        assert g.time == 7
        g.step(9)
        for n in abi.FIELD_NAMES:
            np.testing.assert_array_equal(g.download(n), want[n])
    with runtime.Simulation(cfg) as h:
        h.load_state(snap)
        h.step(9)
        for n in abi.FIELD_NAMES:
            np.testing.assert_array_equal(h.download(n), want[n])
    other = make_case(case, abi.MP_FP64)
    with runtime.Simulation(other) as h:
        with pytest.raises(runtime.MPulseError):
            h.load_state(snap)


@pytest.mark.parametrize("case", ["nonlin_all_short", "nonlin_odd_sizes", "nl_xy", "tma_nonlin_all_short",
                                  "lin_split_cpmlz_gauss"])
def test_kerr_counts(case):
    """mp_kerr_counts: on seeded fields that are non-zero everywhere, every
    medium cell of every E half-step runs the Newton solve once (PLRC-nonlin:
    planes 1..nz inside the medium; fdtd-nl: planes 1..nz+1), each with 1 to
    newton_max_iter iterations; the read resets the counters; the linear
    solver counts nothing."""
    cfg = make_case(case, abi.MP_FP64)
    if case.startswith("tma"):
        cfg.staging = abi.MP_STAGING_TMA
    init = random_fields(cfg, seed=23, smooth=True)
    steps = 3
    with runtime.Simulation(cfg) as g:
        for n, v in init.items():
            g.upload(n, v)
        g.kerr_counts()
        g.step(steps)
        solves, iters = g.kerr_counts()
        assert g.kerr_counts() == (0, 0)
    plane = cfg.nx * cfg.ny
    if cfg.solver == abi.MP_SOLVER_NL:
        want = steps * plane * (cfg.nz + 1)
    elif cfg.solver == abi.MP_SOLVER_PLRC_NONLIN:
        z0, z1 = max(cfg.medium_z0, 1), min(cfg.medium_z1, cfg.nz)
        want = steps * plane * (z1 - z0 + 1)
    else:
        want = 0
    assert solves == want
    assert want <= iters <= want * cfg.newton_max_iter
    if want:
        assert iters > solves  # the solve from |E^n| takes more than one iteration where E changes


def test_plasma_configurations_are_checked():
    """The plasma plug-ins belong to the PLRC solvers and run on the
    global-load kernels; the adjoint of them is not built."""
    cfg = make_case("plasma_nonlin_all_short", abi.MP_FP64)
    cfg.staging = abi.MP_STAGING_TMA
    with pytest.raises(runtime.MPulseError) as e:
        runtime.Simulation(cfg)
    assert e.value.code == abi.MP_ERR_UNSUPPORTED
    bad = make_case("plain_xy", abi.MP_FP64)
    bad.plasma = 1
    with pytest.raises(runtime.MPulseError) as e:
        runtime.Simulation(bad)
    assert e.value.code == abi.MP_ERR_INVALID
    cfg = make_case("plasma_nonlin_all_short", abi.MP_FP64)
    with runtime.Simulation(cfg) as g:
        with pytest.raises(runtime.MPulseError) as e:
            g.adjoint(abi.adjoint_config(abi.MP_OBJ_E2_BOX, (2, 4, 2, 4, 3, 5), 3))
        assert e.value.code == abi.MP_ERR_UNSUPPORTED
    plain = make_case("nonlin_all_short", abi.MP_FP64)
    with runtime.Simulation(plain) as g:
        with pytest.raises(runtime.MPulseError) as e:
            g.download("PlasmaDensity")
        assert e.value.code == abi.MP_ERR_NAME
