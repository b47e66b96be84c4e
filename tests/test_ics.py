"""Seeded initial conditions (no GPU)."""
import math

import numpy as np
import pytest

from cudasph_b200 import ics


@pytest.mark.parametrize("n,xi1", [(1.5, 3.65375), (3.0, 6.89685), (1.0, math.pi)])
def test_lane_emden_first_zero(n, xi1):
    xi, th, dth = ics.lane_emden(n)
    assert abs(xi[-1] - xi1) < 2e-4
    if n == 1.0:  # analytic: theta = sin(xi)/xi
        mid = len(xi) // 2
        assert abs(th[mid] - math.sin(xi[mid]) / xi[mid]) < 1e-8


def test_polytrope_mass_profile_and_seed():
    a = ics.polytrope(4096, seed=5)
    b = ics.polytrope(4096, seed=5)
    c = ics.polytrope(4096, seed=6)
    assert np.array_equal(a["x"], b["x"]) and not np.array_equal(a["x"], c["x"])
    assert abs(a["m"].sum() - 1.0) < 1e-12
    r = np.sqrt(a["x"] ** 2 + a["y"] ** 2 + a["z"] ** 2)
    assert r.max() <= 1.0 + 1e-12
    # enclosed mass at the half-mass radius of an n=1.5 polytrope (R = 1)
    xi, th, dth = ics.lane_emden(1.5)
    mf = -(xi * xi * dth)
    mf /= mf[-1]
    r_half = np.interp(0.5, mf, xi) / xi[-1]
    assert abs(np.mean(r < r_half) - 0.5) < 0.01
    assert np.all(a["u"] > 0) and np.all(a["range"] > 0)


def test_two_star_collision_layout():
    s = ics.two_star_collision(2048, separation=4.0, rel_speed=1.0)
    n = 2048
    assert s["x"].size == 2 * n
    assert abs(s["x"][:n].mean() + 2.0) < 0.05 and abs(s["x"][n:].mean() - 2.0) < 0.05
    assert np.allclose(s["vx"][:n], 0.5) and np.allclose(s["vx"][n:], -0.5)
    assert abs(np.sum(s["m"] * s["vx"])) < 1e-12


def test_cold_sphere_virial_ratio():
    s = ics.cold_sphere(20000, virial=0.1)
    T = 0.5 * np.sum(s["m"] * (s["vx"] ** 2 + s["vy"] ** 2 + s["vz"] ** 2))
    W = 3.0 / 5.0
    assert abs(2 * T / W - 0.1) < 1e-9
    assert np.all(s["u"] == 1e-6)
