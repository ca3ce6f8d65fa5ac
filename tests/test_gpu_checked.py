"""The bounds-checked build (libmpulse_b200_checked.so, MPB_CHECKED=1) on
every forward parity case, every adjoint case (one call and two) and the fused step form's
cases: its step, fused-step, border and adjoint
kernels test each field, history, PLRC, CPML, design and injection-plane
index against the size of its array and make mp_step / mp_adjoint fail with
MP_ERR_BOUNDS instead of touching memory outside an array, so the suites
passing through it show that no case reaches outside its arrays (tiny, odd
and non-tile-multiple grids, overlapping CPML, every solver, boundary, source
and objective, checkpoint schedules).  The library is loaded once per
process, so each suite runs in a child process."""
import os
import subprocess
import sys

import pytest

from mpulse_b200 import build

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("suite", ["test_gpu_parity.py", "test_gpu_adjoint.py", "test_gpu_adjoint_record.py",
                                   "test_gpu_fused.py"])
def test_suite_passes_through_the_checked_build(suite):
    assert os.path.exists(build.LIB_CHECKED), "build the checked library: python -m mpulse_b200.build --checked"
    env = dict(os.environ, MPULSE_B200_LIB=build.LIB_CHECKED)
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", "-m", "gpu",
                        os.path.join(ROOT, "tests", suite)],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout
