"""Generates the golden fixtures of tests/golden/ by running the reference
build (oracle/_ref/mpulse_ref: MPulse's own sources compiled by
oracle/Makefile, -O2 -ffp-contract=off) on seeded inputs.

    make -C oracle ref && python tests/golden/make_golden.py

Each fixture holds the mp_config (as JSON), the seed of the initial fields
(tests/cases.random_fields), a SHA-256 of those fields, the number of steps
and the reference's fields after those steps, in the plane layout of
include/mpulse_b200.h.  The workload fixtures keep only one x-z slice per field
and the total field energy, to stay small.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mpulse_b200 import abi, configs  # noqa: E402
from oracle import pyoracle  # noqa: E402
from tests.cases import CASES, make_case, random_fields  # noqa: E402

GOLDEN_N = (10, 8, 14)
GOLDEN_STEPS = 30


def init_digest(init: dict) -> str:
    h = hashlib.sha256()
    for n in abi.FIELD_NAMES:
        h.update(np.ascontiguousarray(init[n], dtype=np.float64).tobytes())
    return h.hexdigest()


def small_case(name: str) -> abi.Config:
    cfg = make_case(name, abi.MP_FP64)
    spec = CASES[name]
    if "n" not in spec:
        cfg.nx, cfg.ny, cfg.nz = GOLDEN_N
        if spec.get("medium"):
            cfg.medium_z0, cfg.medium_z1 = 5, 11
        for q in range(cfg.n_sources):
            cfg.sources[q].distance = 6
    return cfg


def case_seed(name: str) -> int:
    return sum(map(ord, name)) % 997


def case_names(cfg: abi.Config) -> tuple:
    """The grids a fixture keeps: the fields, and the plasma plug-ins' state."""
    return abi.FIELD_NAMES + (abi.PLASMA_NAMES if (cfg.plasma or cfg.plasma_current) else ())


def write_case(name: str):
    cfg = small_case(name)
    seed = case_seed(name)
    init = random_fields(cfg, seed=seed)
    names = case_names(cfg)
    out, timing = pyoracle.run_reference(cfg, GOLDEN_STEPS, init, names=names)
    np.savez_compressed(
        os.path.join(HERE, f"case_{name}.npz"),
        config=json.dumps(abi.config_to_dict(cfg)), seed=seed, steps=GOLDEN_STEPS,
        init_sha256=init_digest(init), **{n: out[n] for n in names})
    print(name, timing["seconds"])


def workload_fixture(name: str, cfg: abi.Config, steps: int, init: dict | None, start_time: int = 0):
    """Reference run of a reduced workload; keeps the x-z slice at y = ny/2 and
    the energy sum(E^2 + B^2) over the interior planes."""
    if start_time:
        raise ValueError("the reference starts at time 0")
    out, timing = pyoracle.run_reference(cfg, steps, init)
    j = cfg.ny // 2
    energy = float(sum(np.sum(out[n][1:-1] ** 2) for n in abi.FIELD_NAMES))
    np.savez_compressed(
        os.path.join(HERE, f"workload_{name}.npz"),
        config=json.dumps(abi.config_to_dict(cfg)), steps=steps, slice_y=j, energy=energy,
        has_init=init is not None, **{n: out[n][:, j, :] for n in abi.FIELD_NAMES})
    print(name, timing["seconds"], "energy", energy)


def main():
    only = sys.argv[1:]  # case names to (re)write; default: all cases and workloads
    for name in sorted(CASES):
        if not only or name in only:
            write_case(name)
    if only:
        return
    # the vacuum pulse workload at full size (64^3, 400 steps)
    c1 = configs.c1_vacuum_pulse(abi.MP_FP64)
    workload_fixture("c1_vacuum_pulse_64", c1, 400, configs.c1_initial_fields(c1))
    # the linear PLRC workload reduced to 24 x 24 x 128 with the same z layout
    c2 = configs.c2_linear_plrc(abi.MP_FP64, n=128)
    c2.nx = c2.ny = 24
    workload_fixture("c2_linear_plrc_24x24x128", c2, 600, None)
    # the PLRC + Kerr + focused short pulse workload reduced to 48 x 48 x 96
    c3 = configs.c3_plrc_kerr(abi.MP_FP64, nx=48, ny=48, nz=96, medium_z0=40, focus_z=60, src_d=16, chi=0.01)
    c3.sources[0].waist = 0.6
    c3.sources[0].t_shift = 2.0 * c3.sources[0].length + 1.0
    workload_fixture("c3_plrc_kerr_48x48x96", c3, 300, None)


if __name__ == "__main__":
    main()
