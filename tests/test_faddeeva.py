"""The oracle's Faddeeva evaluator (Weideman's expansion, N = 40) against
scipy.special.wofz in the upper half plane, where the short-pulse fields use
it (shortpulsefunctions.cpp:77-91 only call it with Im z >= 0)."""
import numpy as np
from scipy.special import wofz

from oracle import pyoracle


def test_faddeeva_upper_half_plane():
    rng = np.random.default_rng(0)
    for scale in (0.01, 0.3, 1.0, 3.0, 10.0, 100.0):
        z = (rng.uniform(-1, 1, 4000) + 1j * rng.uniform(0, 1, 4000)) * scale
        w = pyoracle.faddeeva(z)
        ref = wofz(z)
        assert np.max(np.abs(w - ref) / np.abs(ref)) < 5e-14


def test_faddeeva_special_values():
    w = pyoracle.faddeeva(np.array([0.0 + 0.0j, 1j, 2j]))
    np.testing.assert_allclose(w.real, wofz(np.array([0j, 1j, 2j])).real, rtol=1e-14)
    assert abs(w[0] - 1.0) < 1e-14
