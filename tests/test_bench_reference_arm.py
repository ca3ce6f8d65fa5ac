"""bench.py's reference arm on the host: it runs the reference build (the
MPulse sources compiled by oracle/Makefile) on the headline workload split
into z-slab processes and prints one JSON line with the contract's keys.  No
GPU is involved."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = [os.path.join(ROOT, "oracle", "_ref", n) for n in ("mpulse_ref_fast", "mpulse_ref")]


@pytest.mark.skipif(not any(os.path.exists(p) for p in REF), reason="reference build absent (make -C oracle ref)")
def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.strip().splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "steps", "warmup", "ms_per_step", "higher_is_better", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"


@pytest.mark.skipif(not any(os.path.exists(p) for p in REF), reason="reference build absent (make -C oracle ref)")
def test_reference_arm_config_is_the_workload_of_the_gpu_arm():
    """Both arms name the same workload object in `config` (the same grid,
    medium, CPML, source and dt); only `parallelism` and the state differ."""
    sys.path.insert(0, ROOT)
    import bench
    from mpulse_b200 import abi
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads([ln for ln in r.stdout.strip().splitlines() if ln.startswith("{")][0])
    assert d["config"] == bench.workload_config_keys(bench.bench_config(abi.MP_FP32))
    assert d["cpu_baseline"]["same_config"] is True


@pytest.mark.skipif(not os.path.exists(REF[1]), reason="reference build absent (make -C oracle ref)")
def test_slab_boundary_whole_grid_equals_single_xy_periodic_and_slabs_cover_the_grid():
    """The harness's slab_xy_periodic boundary (the reference's timed form):
    one slab over the whole grid is MPulse's single_xy_periodic run bit for
    bit, and a split into z-slabs holds every interior cell exactly once."""
    sys.path.insert(0, ROOT)
    from mpulse_b200 import abi
    from oracle import pyoracle
    from tests.cases import make_case, random_fields
    cfg = make_case("nonlin_all_short", abi.MP_FP64)
    init = random_fields(cfg, seed=5, smooth=True)
    whole, t1 = pyoracle.run_reference(cfg, 6, init_fields=init, binary=REF[1])
    slab, t2 = pyoracle.run_reference(cfg, 6, init_fields=init, binary=REF[1],
                                      boundary=f"slab_xy_periodic {{ z0 1 z1 {cfg.nz} }}")
    for n in abi.FIELD_NAMES:
        assert np.array_equal(whole[n], slab[n]), n
    assert t1["cells"] == t2["cells"] == cfg.nx * cfg.ny * cfg.nz
    cells = 0
    for z0, z1 in ((1, 9), (10, 19), (20, cfg.nz)):
        _, t = pyoracle.run_reference(cfg, 1, init_fields=init, binary=REF[1], names=(),
                                      boundary=f"slab_xy_periodic {{ z0 {z0} z1 {z1} }}")
        assert t["low"][2] == z0 - 1 and t["high"][2] == z1 + 1
        cells += t["cells"]
    assert cells == cfg.nx * cfg.ny * cfg.nz
