"""Seeded synthetic initial conditions for the SPH + self-gravity step.

The reference ships no input (its one initial condition, ``init.bin.60k.gz``,
is missing from the tree), so every workload here is generated:

* :func:`polytrope` -- an n-polytrope (Lane-Emden) star of mass M and radius R,
  G = 1, particles placed by radially stretching a randomly rotated cubic
  lattice so that the enclosed-mass profile matches the polytrope; thermal
  energy u = K rho^(1/n) / (gamma - 1) from P = K rho^(1 + 1/n).
* :func:`two_star_collision` -- two polytropes head on.
* :func:`cold_sphere` -- a uniform-density sphere with isotropic velocities at a
  given virial ratio 2T/|W|.

Each returns a dict of float64 numpy arrays in the reference's particle layout
(``CUDAsph.h:50-68``): x, y, z, vx, vy, vz, m, range (= 2h), u, mu, plus ``dt``
(0: the first step starts with a half kick).  Initial smoothing ranges come
from the analytic density and the target neighbour number; the h solve
refines them.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["lane_emden", "polytrope", "two_star_collision", "cold_sphere", "initial_range"]


def lane_emden(n: float, dxi: float = 1e-4):
    """Integrate theta'' + 2 theta'/xi + theta^n = 0 with RK4 from the centre.

    Returns (xi, theta, dtheta) sampled up to the first zero xi_1 (the last
    sample is interpolated onto theta = 0).
    """
    xi0 = 1e-6
    th = 1.0 - xi0 * xi0 / 6.0
    dth = -xi0 / 3.0

    def f(x, t, d):
        tp = max(t, 0.0)
        return d, -(tp ** n) - 2.0 * d / x

    xs, ts, ds = [xi0], [th], [dth]
    x = xi0
    while th > 0:
        k1 = f(x, th, dth)
        k2 = f(x + 0.5 * dxi, th + 0.5 * dxi * k1[0], dth + 0.5 * dxi * k1[1])
        k3 = f(x + 0.5 * dxi, th + 0.5 * dxi * k2[0], dth + 0.5 * dxi * k2[1])
        k4 = f(x + dxi, th + dxi * k3[0], dth + dxi * k3[1])
        th_n = th + dxi / 6.0 * (k1[0] + 2 * k2[0] + 2 * k3[0] + k4[0])
        dth_n = dth + dxi / 6.0 * (k1[1] + 2 * k2[1] + 2 * k3[1] + k4[1])
        if th_n <= 0:
            frac = th / (th - th_n)
            x = x + frac * dxi
            xs.append(x)
            ts.append(0.0)
            ds.append(dth + frac * (dth_n - dth))
            break
        x += dxi
        th, dth = th_n, dth_n
        xs.append(x)
        ts.append(th)
        ds.append(dth)
    return np.array(xs), np.array(ts), np.array(ds)


def _lattice_ball(n: int, rng: np.random.Generator) -> np.ndarray:
    """The n points of a randomly rotated and offset cubic lattice nearest the
    origin, scaled into the unit ball, ordered by radius."""
    k = int(math.ceil((n * 6.0 / math.pi) ** (1.0 / 3.0))) + 4
    g = np.arange(-k, k + 1, dtype=np.float64)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    pts += rng.uniform(-0.5, 0.5, size=3)
    # random rotation (QR of a Gaussian matrix)
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    pts = pts @ q.T
    rad = np.sqrt((pts * pts).sum(axis=1))
    tie = rng.random(rad.shape[0]) * 1e-9
    order = np.argsort(rad + tie, kind="stable")[:n]
    pts = pts[order]
    rad = rad[order]
    return pts, rad


def initial_range(rho: np.ndarray, m: np.ndarray, n_ngb: float) -> np.ndarray:
    """range = 2h holding ~n_ngb particles: (4 pi / 3) range^3 rho = n_ngb m."""
    return (3.0 * n_ngb * m / (4.0 * math.pi * np.maximum(rho, 1e-300))) ** (1.0 / 3.0)


def polytrope(n_part: int, n_poly: float = 1.5, M: float = 1.0, R: float = 1.0, gamma: float = 5.0 / 3.0,
              n_ngb: float = 50.0, seed: int = 12345, mu: float = 0.62, u_jitter: float = 0.0,
              lattice_jitter: float = 0.05):
    """An n-polytrope of mass M and radius R (G = 1) with n_part equal-mass particles."""
    rng = np.random.default_rng(seed)
    xi, th, dth = lane_emden(n_poly)
    xi1 = xi[-1]
    mfrac = -(xi * xi * dth)
    mfrac = mfrac / mfrac[-1]
    mfrac[0] = 0.0
    # central density and K from M, R (Chandrasekhar's polytrope relations, G = 1)
    a = R / xi1
    w1 = -(xi1 * xi1 * dth[-1])
    rho_c = M / (4.0 * math.pi * a ** 3 * w1)
    K = 4.0 * math.pi * a * a * rho_c ** (1.0 - 1.0 / n_poly) / (n_poly + 1.0)

    pts, rad = _lattice_ball(n_part, rng)
    dirs = pts / np.maximum(rad, 1e-300)[:, None]
    # stretch: the k-th particle by radius encloses mass fraction (k + 0.5) / N
    target = (np.arange(n_part) + 0.5) / n_part
    r_new = np.interp(target, mfrac, xi) * a
    # keep the lattice's angular pattern; jitter the radial assignment slightly
    if lattice_jitter > 0:
        sp = (1.0 / n_part) ** (1.0 / 3.0) * R
        r_new = r_new + rng.uniform(-lattice_jitter, lattice_jitter, n_part) * sp * 0.1
        r_new = np.clip(r_new, 0.0, R)
    pos = dirs * r_new[:, None]
    theta = np.interp(r_new / a, xi, th)
    rho = rho_c * np.maximum(theta, 0.0) ** n_poly
    rho_floor = rho_c * 1e-4
    rho = np.maximum(rho, rho_floor)
    m = np.full(n_part, M / n_part)
    u = K * rho ** (1.0 / n_poly) / (gamma - 1.0)
    if u_jitter > 0:
        u = u * (1.0 + rng.uniform(-u_jitter, u_jitter, n_part))
    rng_ = initial_range(rho, m, n_ngb)
    z = np.zeros(n_part)
    return {
        "x": pos[:, 0].copy(), "y": pos[:, 1].copy(), "z": pos[:, 2].copy(),
        "vx": z.copy(), "vy": z.copy(), "vz": z.copy(),
        "m": m, "range": rng_, "u": u, "mu": np.full(n_part, mu),
        "dt": 0.0,
    }


def two_star_collision(n_each: int, separation: float = 4.0, rel_speed: float = 1.0, n_poly: float = 1.5,
                       n_ngb: float = 64.0, seed: int = 12345, mu: float = 0.62):
    """Two equal n-polytropes (M = R = 1) with centres `separation` apart on x,
    approaching head on at relative speed `rel_speed` (+-rel_speed/2 each)."""
    a = polytrope(n_each, n_poly=n_poly, n_ngb=n_ngb, seed=seed, mu=mu)
    b = polytrope(n_each, n_poly=n_poly, n_ngb=n_ngb, seed=seed + 1, mu=mu)
    out = {}
    for k in ("x", "y", "z", "vx", "vy", "vz", "m", "range", "u", "mu"):
        out[k] = np.concatenate([a[k], b[k]])
    out["x"][:n_each] -= 0.5 * separation
    out["x"][n_each:] += 0.5 * separation
    out["vx"][:n_each] += 0.5 * rel_speed
    out["vx"][n_each:] -= 0.5 * rel_speed
    out["dt"] = 0.0
    return out


def cold_sphere(n_part: int, virial: float = 0.1, M: float = 1.0, R: float = 1.0, u0: float = 1e-6,
                n_ngb: float = 50.0, seed: int = 12345, mu: float = 0.62):
    """Uniform-density sphere with isotropic Gaussian velocities scaled so that
    2T/|W| = virial, W = -3 G M^2 / (5 R)."""
    rng = np.random.default_rng(seed)
    r = R * rng.random(n_part) ** (1.0 / 3.0)
    v = rng.standard_normal((n_part, 3))
    d = v / np.linalg.norm(v, axis=1)[:, None]
    pos = d * r[:, None]
    vel = rng.standard_normal((n_part, 3))
    vel -= vel.mean(axis=0)
    m = np.full(n_part, M / n_part)
    T = 0.5 * (m[:, None] * vel * vel).sum()
    W = 3.0 * M * M / (5.0 * R)
    vel *= math.sqrt(virial * W / (2.0 * T))
    rho = np.full(n_part, 3.0 * M / (4.0 * math.pi * R ** 3))
    return {
        "x": pos[:, 0].copy(), "y": pos[:, 1].copy(), "z": pos[:, 2].copy(),
        "vx": vel[:, 0].copy(), "vy": vel[:, 1].copy(), "vz": vel[:, 2].copy(),
        "m": m, "range": initial_range(rho, m, n_ngb), "u": np.full(n_part, u0), "mu": np.full(n_part, mu),
        "dt": 0.0,
    }
