"""Closed-form known answers for the checks.

TEST INFRASTRUCTURE: used by tests/ only.  The product (cudasph_b200) never
imports it.

softened_pair: what one source puts on a target at separation r under the
two softenings of the gravity path.  The reference's spline softening
(sph_grav_kernel.cu:32-105) is the M4 cubic spline's softened force and
potential with support `range` = 2h, applied with half contributions at the
target's and at the source's range for the force and at the target's range
alone for the potential.  Here the softened law is written from its published
closed form (Hernquist & Katz 1989; Price & Monaghan 2007) with exact rational
coefficients in q = r / h.  So it pins the reference's 12-decimal constants,
and the oracle and GPU kernels that carry them, to the physics: they agree to
about 1e-12.
"""
from __future__ import annotations

import math


def spline_force_shape(q: float) -> float:
    """f(q) with |a| = G m f(q) / h^2 for one source of mass m at r = q h."""
    if q < 1.0:
        return 4.0 / 3.0 * q - 6.0 / 5.0 * q ** 3 + 0.5 * q ** 4
    if q < 2.0:
        return 8.0 / 3.0 * q - 3.0 * q ** 2 + 6.0 / 5.0 * q ** 3 - q ** 4 / 6.0 - 1.0 / (15.0 * q ** 2)
    return 1.0 / q ** 2


def spline_potential_shape(q: float) -> float:
    """phi(q) with potential = G m phi(q) / h for one source of mass m at r = q h."""
    if q < 1.0:
        return 2.0 / 3.0 * q ** 2 - 0.3 * q ** 4 + 0.1 * q ** 5 - 1.4
    if q < 2.0:
        return 4.0 / 3.0 * q ** 2 - q ** 3 + 0.3 * q ** 4 - q ** 5 / 30.0 - 1.6 + 1.0 / (15.0 * q)
    return -1.0 / q


def _spline_k(r: float, rng: float) -> float:
    """K(r, range) with a = -G m K d, d = x_target - x_source (r > 0; the r -> 0 limit at r = 0)."""
    if r >= rng:
        return 1.0 / r ** 3
    h = 0.5 * rng
    if r == 0.0:
        return 4.0 / 3.0 / h ** 3
    return spline_force_shape(r / h) / (h * h * r)


def softened_pair(r: float, range_t: float, range_s: float, soft_mode: int, eps: float) -> tuple[float, float]:
    """(K, P) of a source at separation r from the target: the target's
    acceleration is -G m_s K (x_t - x_s) and its potential G m_s P.
    soft_mode 0: spline softening at the ranges of target and source (half
    contributions for the force, the target's range for the potential), as
    sph_grav_kernel.cu:32-105 applies it; 1: Plummer with length eps."""
    if soft_mode == 1:
        s2 = r * r + eps * eps
        return s2 ** -1.5, -1.0 / math.sqrt(s2)
    if r >= range_t and r >= range_s:
        if r == 0.0:
            return 0.0, 0.0
        return 1.0 / r ** 3, -1.0 / r
    k = 0.5 * _spline_k(r, range_t) + 0.5 * _spline_k(r, range_s)
    if r < range_t:
        h = 0.5 * range_t
        p = spline_potential_shape(r / h) / h
    else:
        p = -1.0 / r
    return k, p


def two_body(r: float, ranges=(0.2, 0.3), masses=(0.7, 1.3), soft_mode: int = 0, eps: float = 0.0, G: float = 1.0):
    """Two particles at separation r along (2, -1, 2) / 3 and the closed-form
    gravity on each (every particle also meets itself: no force, its own
    potential term), as arrays pos (2, 3), m (2), range (2), acc (2, 3),
    phi (2)."""
    import numpy as np
    x0 = np.array([0.1, -0.2, 0.3])
    pos = np.stack([x0, x0 + r * np.array([2.0, -1.0, 2.0]) / 3.0])
    m = np.array(masses, float)
    rng = np.array(ranges, float)
    acc = np.zeros((2, 3))
    phi = np.zeros(2)
    for t, s in ((0, 1), (1, 0)):
        d = pos[t] - pos[s]
        rr = float(np.sqrt(np.sum(d * d)))  # the separation the stored positions hold
        k, p = softened_pair(rr, rng[t], rng[s], soft_mode, eps)
        _, p_self = softened_pair(0.0, rng[t], rng[t], soft_mode, eps)
        acc[t] = -G * m[s] * k * d
        phi[t] = G * (m[s] * p + m[t] * p_self)
    return pos, m, rng, acc, phi
