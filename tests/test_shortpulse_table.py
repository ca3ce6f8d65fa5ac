"""The short-pulse closed form of the oracle (the one the device kernels
restate) against the reference's own short-pulse test program
(test/testshortpulse.cpp): Efunc and Bfunc with setParam(length 1e6, width 2,
om0 2, Shift 0, Phase 0, amp 1, eps 1) on a 51 x 80 grid of (x, t) at
y = z = 0 (tests/golden/shortpulse_table.npz, made by
tests/golden/make_shortpulse_table.py).  The program prints six significant
digits, so every value agrees to 1e-5 of itself plus 1e-6 of the column's
largest magnitude."""
import os

import numpy as np
import pytest

from oracle import pyoracle

TABLE = os.path.join(os.path.dirname(__file__), "golden", "shortpulse_table.npz")


def test_oracle_matches_reference_short_pulse_table():
    d = np.load(TABLE)
    x, t, v = d["x"], d["t"], d["values"]
    length, width, om0, phase, eps = d["params"]
    scale = np.abs(v).max(axis=(0, 1))
    got = np.array([[pyoracle.short_pulse(length, width, om0, phase, eps, xa, 0.0, 0.0, tb) for tb in t] for xa in x])
    tol = 1e-5 * np.abs(v) + 1e-6 * scale
    assert np.all(np.abs(got - v) <= tol), float(np.max(np.abs(got - v) - tol))
    # Bx vanishes on the y = 0 line (its terms carry d tp / dy = -y / (c q))
    assert np.all(got[..., 2:4] == 0.0)


@pytest.mark.parametrize("q", [0, 4])
def test_table_is_not_trivial(q):
    """The pulse crosses the table: Re Efunc and Re Bfunc(by) reach the field
    scale and change sign along t."""
    v = np.load(TABLE)["values"][..., q]
    assert np.abs(v).max() > 1.0
    assert (v > 0).any() and (v < 0).any()
