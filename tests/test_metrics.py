"""Integrated quantities (camr_b200/metrics.py) and their drift."""
import numpy as np

from camr_b200 import metrics
from camr_b200 import problems as P


def test_integrated_quantities_are_volume_weighted_sums():
    n = (8, 6, 4)
    s = P.random_smooth(n, seed=5)
    dx = (0.5, 0.25, 0.125)
    q = metrics.integrated_quantities(s, dx)
    vol = 0.5 * 0.25 * 0.125
    assert np.isclose(q["mass"], s[0].sum() * vol, rtol=1e-14)
    assert np.isclose(q["rho_E"], s[4].sum() * vol, rtol=1e-14)
    kin = 0.5 * (s[1] ** 2 + s[2] ** 2 + s[3] ** 2) / s[0]
    assert np.isclose(q["kineng"], kin.sum() * vol, rtol=1e-14)


def test_drift_of_a_shifted_state_is_zero_and_of_a_scaled_one_is_not():
    n = (8, 6, 4)
    s = P.random_smooth(n, seed=6)
    dx = (0.1, 0.1, 0.1)
    q0 = metrics.integrated_quantities(s, dx)
    # a periodic shift conserves every sum
    q1 = metrics.integrated_quantities(np.roll(s, 3, axis=3), dx)
    d = metrics.drift(q0, q1)
    assert abs(d["mass_rel"]) < 1e-14 and abs(d["rho_E_rel"]) < 1e-14
    assert all(abs(v) < 1e-12 for v in d["momentum_rel"].values())
    t = s.copy()
    t[0] *= 1.001
    d = metrics.drift(q0, metrics.integrated_quantities(t, dx))
    assert np.isclose(d["mass_rel"], 1e-3, rtol=1e-9)
