"""The bounds-checked build (libmpulse_b200_checked.so, MPB_CHECKED=1) on
every forward parity case: its step kernels test each field, PLRC, CPML and
injection-plane index against the size of its array and make mp_step fail
with MP_ERR_BOUNDS instead of touching memory outside an array, so the
parity suite passing through it shows that no case reaches outside its
arrays (tiny, odd and non-tile-multiple grids, overlapping CPML, every
solver, boundary and source).  The library is loaded once per process, so the
suite runs in a child process."""
import os
import subprocess
import sys

import pytest

from mpulse_b200 import build

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_parity_suite_passes_through_the_checked_build():
    assert os.path.exists(build.LIB_CHECKED), "build the checked library: python -m mpulse_b200.build --checked"
    env = dict(os.environ, MPULSE_B200_LIB=build.LIB_CHECKED)
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", "-m", "gpu",
                        os.path.join(ROOT, "tests", "test_gpu_parity.py")],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout
