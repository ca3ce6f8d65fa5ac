"""Loading of the golden fixtures made by tests/golden/make_golden.py."""
from __future__ import annotations

import glob
import hashlib
import json
import os

import numpy as np

from mpulse_b200 import abi, configs
from tests.cases import random_fields

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def case_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "case_*.npz")))


def workload_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "workload_*.npz")))


def load(path):
    """A fixture and its mp_config.  Fixtures written before a field was added
    to mp_config lack it and get its default; the ABI version is the
    library's."""
    d = np.load(path)
    cfg = abi.config_from_dict(json.loads(str(d["config"])))
    cfg.abi_version = abi.MP_ABI_VERSION
    return d, cfg


def case_init(d, cfg):
    init = random_fields(cfg, seed=int(d["seed"]))
    h = hashlib.sha256()
    for n in abi.FIELD_NAMES:
        h.update(np.ascontiguousarray(init[n], dtype=np.float64).tobytes())
    assert h.hexdigest() == str(d["init_sha256"]), "seeded initial fields changed"
    return init


def workload_init(path, cfg):
    name = os.path.basename(path)
    if name.startswith("workload_c1_"):
        return configs.c1_initial_fields(cfg)
    return None
