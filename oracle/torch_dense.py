"""Dense O(N^2) FP64 PyTorch restatement of one step, differentiable by autograd.

TEST INFRASTRUCTURE: the reference the hand-written adjoint kernels are checked
against (and a second, independent forward check of the oracle).  It builds
every pair explicitly (N x N tensors), so it is for small N only.

It follows the same reference loops as sph_oracle.c -- predictor and kick
(step.cpp:38-61,128-134), smoothing-length solve (dev_solve_range.cu:17-172),
density (dev_density_loop.cu:29-86), EOS (dev_compute_pressure.cu:83-96),
artificial viscosity (dev_art_visc.cu:8-32), hydro (dev_hydro_dots.cu:25-84)
with the j-side of sph_accelerations.cpp:106-114, Plummer gravity, and
compute_timestep.cpp:3-25 -- with these differentiation conventions:

* the smoothing range is the root of F_i(w) = sum_j ig(2 r_ij / w) - N
  (found without gradient), re-attached so that autograd sees the implicit
  derivative dw/dx = -(dF/dx) / (dF/dw);
* max (signal speed) and min (timestep) pass the gradient to the arg-max /
  arg-min, as a discrete derivative of those operations does.
"""
from __future__ import annotations

import math

import torch

IPI = 0.318309886183791
PI = 3.141592653589793


def _w(u):
    u2 = u * u
    a = IPI * (1 - 1.5 * u2 + 0.75 * u2 * u)
    t = (2 - u).clamp(min=0)
    b = IPI * 0.25 * t * t * t
    return torch.where(u < 1, a, torch.where(u < 2, b, torch.zeros_like(u)))


def _dw(u):
    us = torch.where(u < 1, torch.ones_like(u), u)  # safe divisor for the outer branch
    a = IPI * (-3 + 2.25 * u)
    t = (2 - u).clamp(min=0)
    b = -IPI * 0.75 * t * t / us
    return torch.where(u < 1, a, torch.where(u < 2, b, torch.zeros_like(u)))


def _dwdh(u):
    u2 = u * u
    a = IPI * (-3 + 7.5 * u2 - 4.5 * u2 * u)
    b = IPI * (-6 + 12 * u - 7.5 * u2 + 1.5 * u2 * u)
    return torch.where(u < 1, a, torch.where(u < 2, b, torch.zeros_like(u)))


def _dphidh(u):
    u2 = u * u
    a = 1.4 - 2 * u2 + 1.5 * u2 * u2 - 0.6 * u2 * u2 * u
    b = 1.6 - 4 * u2 + 4 * u2 * u - 1.5 * u2 * u2 + 0.2 * u2 * u2 * u
    return torch.where(u < 1, a, torch.where(u < 2, b, torch.zeros_like(u)))


def _iw(x):
    x3 = x * x * x
    a = 4 * (x3 / 3.0 - 0.3 * x3 * x * x + 0.125 * x3 * x3)
    b = 4 * (-1.0 / 60 + 2.0 / 3 * x3 - 0.75 * x3 * x + 0.3 * x3 * x * x - x3 * x3 / 24.0)
    return torch.where(x < 0, torch.zeros_like(x), torch.where(x < 1, a, torch.where(x < 2, b, torch.ones_like(x))))


def _ig(u):
    return _iw(4.0 * (1.0 - (u - 1.0).abs()))


def _diw(x):
    return 4.0 * PI * x * x * _w(x)


def _dig(u):
    us = torch.where(u > 0, u, torch.ones_like(u))
    a = 4.0 / us * _diw(4.0 * u)
    b = -4.0 / us * _diw(4.0 * (2 - u))
    return torch.where(u <= 0, torch.zeros_like(u), torch.where(u < 1, a, torch.where(u < 2, b, torch.zeros_like(u))))


def _digdh(u):
    a = 4.0 * u * _diw(4.0 * u)
    b = -4.0 * u * _diw(4.0 * (2 - u))
    return torch.where(u <= 0, torch.zeros_like(u), torch.where(u < 1, a, torch.where(u < 2, b, torch.zeros_like(u))))


def _pairs(x):
    d = x[:, None, :] - x[None, :, :]          # d_ij = x_i - x_j
    r2 = (d * d).sum(-1)
    pos = r2 > 0
    r = torch.sqrt(torch.where(pos, r2, torch.ones_like(r2))) * pos
    return d, r2, r


def solve_h(x, w0, n_target, rel_err=1e-12, iters=200):
    """Smoothing ranges (the root of the smooth count), then re-attached with
    the implicit derivative.  Safeguarded Newton on each particle."""
    with torch.no_grad():
        d, r2, r = _pairs(x)
        w = w0.clone()
        lo = torch.zeros_like(w)
        hi = torch.full_like(w, float("inf"))
        for _ in range(iters):
            u = 2 * r / w[:, None]
            m = r2 < (w * w)[:, None]
            f = (_ig(u) * m).sum(1) - n_target
            g = -(_digdh(u) * m).sum(1) / w
            lo = torch.where(f < 0, torch.maximum(lo, w), lo)
            hi = torch.where(f >= 0, torch.minimum(hi, w), hi)
            step = torch.where(g != 0, f / g, torch.where(f < 0, -w, w))
            wn = w - step
            bad = ~((wn > lo) & (wn < hi))
            mid = torch.where(torch.isfinite(hi), 0.5 * (lo + hi), 2 * w)
            wn = torch.where(bad, mid, wn)
            if torch.all((wn - w).abs() <= rel_err * w):
                w = wn
                break
            w = wn
    # re-attach: w = w* - F(w*, x) / F_w(w*, x).detach()
    d, r2, r = _pairs(x)
    u = 2 * r / w[:, None]
    m = r2 < (w * w)[:, None]
    F = (_ig(u) * m).sum(1) - n_target
    Fw = (-(_digdh(u) * m).sum(1) / w).detach()
    return w.detach() - F / Fw


def density(x, v, m, w):
    d, r2, r = _pairs(x)
    msk = (r2 < (w * w)[:, None]).to(x.dtype)
    h = 0.5 * w
    u = r / h[:, None]
    mj = m[None, :]
    rho = (mj * _w(u) * msk).sum(1) / h ** 3
    om = (mj * _dwdh(u) * msk).sum(1)
    ps = (mj * _dphidh(u) * msk).sum(1)
    sdig = -(_digdh(u) * msk).sum(1)
    dv = v[:, None, :] - v[None, :, :]
    wt = mj * _dw(u) * msk
    div = (wt * (d * dv).sum(-1)).sum(1)
    cr = torch.cross(d, dv, dim=-1)
    c = (wt[..., None] * cr).sum(1)
    om = om / h ** 3 / sdig
    ps = ps / h / sdig
    div = div / rho / h ** 5
    curl = torch.sqrt((c * c).sum(-1)) / rho / h ** 5
    return rho, div, curl, om, ps


DENSITY_UNIT = 5.89994031541978
ENERGY_UNIT = 1.90698842928778e+15
PRESSURE_UNIT = 1.1251117914994e+16
AMU = 1.66054e-24
BOLTZMANN = 1.380658e-16
RAD_CONST = 7.56591414984829e-15


def pressure(rho, u, mu, eos_mode, gamma):
    if eos_mode == 0:
        return (gamma - 1) * rho * u
    dens = rho * DENSITY_UNIT
    en = u * ENERGY_UNIT
    mm = mu * AMU
    tb = 1.0e6
    r = -dens * (en / (tb * tb)) / (RAD_CONST * tb * tb)
    q = (BOLTZMANN / RAD_CONST) / (gamma - 1) * dens / (((mm * tb) * tb) * tb)
    with torch.no_grad():
        x = torch.minimum(-r / q, (-r) ** 0.25)
        for _ in range(100):
            x = x - (x ** 4 + q * x + r) / (4 * x ** 3 + q)
    # implicit derivative of the positive root of x^4 + q x + r = 0
    xs = x.detach()
    x = xs - (xs ** 4 + q * xs + r) / (4 * xs ** 3 + q).detach()
    T = tb * x
    pg = dens * ((BOLTZMANN * T) / mm)
    pr = (((RAD_CONST / 3.0 * T) * T) * T) * T
    return (pg + pr) / PRESSURE_UNIT


def hydro(x, v, m, w, rho, P, div, curl, om, ps, p):
    d, r2, r = _pairs(x)
    msk = r2 < (w * w)[:, None]
    mf = msk.to(x.dtype)
    hh = 0.5 * w
    u = r / hh[:, None]
    dv = v[:, None, :] - v[None, :, :]
    drdv = (d * dv).sum(-1)
    gam, alpha, beta = p["gamma"], p["alpha"], p["beta"]
    c = torch.sqrt(gam * P / rho)
    ci, cj = c[:, None], c[None, :]
    rs = torch.where(r > 0, r, torch.ones_like(r))
    neg = drdv < 0
    vs = ci + cj - torch.where(neg, beta * drdv / rs, torch.zeros_like(r))
    mu_ = drdv / ((ci + cj) * rs)
    bi = div.abs() / (div.abs() + curl + 0.0001 * c / (0.5 * w))
    bal = bi[:, None] + bi[None, :]
    mu_ = mu_ * bal
    prho2 = P / rho ** 2
    visc = torch.where(neg, (prho2[:, None] + prho2[None, :]) * (-alpha * mu_ + beta * mu_ * mu_),
                       torch.zeros_like(r))
    vsig = torch.where(msk, vs, torch.full_like(vs, -float("inf"))).max(1).values
    dwu, digu = _dw(u), _dig(u)
    h5 = (hh ** 5)[:, None]
    h2 = (hh ** 2)[:, None]
    psi_i = ps * p["use_psi"]
    acc = (prho2[:, None] + 0.5 * visc) * dwu / h5
    acc = acc - (prho2[:, None] * om[:, None] + 0.5 * psi_i[:, None]) / m[None, :] * digu / h2
    acc = acc * mf
    a_i = -((m[None, :] * acc)[..., None] * d).sum(1)
    # j-side: a_j += m_i acc_ij d_ij  ->  for particle k: sum_i m_i acc_ik d_ik
    a_j = ((m[:, None] * acc)[..., None] * d).sum(0)
    ud = m[None, :] * (prho2[:, None] + 0.5 * visc) * dwu / h5 - prho2[:, None] * om[:, None] * digu / h2
    du = (ud * drdv * mf).sum(1)
    return a_i + a_j, du, vsig


def gravity_plummer(x, m, eps, G=1.0):
    d = x[None, :, :] - x[:, None, :]          # x_j - x_i
    s2 = (d * d).sum(-1) + eps * eps
    inv = s2 ** -0.5
    g = (m[None, :, None] * d * (inv ** 3)[..., None]).sum(1)
    phi = -(m[None, :] * inv).sum(1)
    return G * g, G * phi


def timestep(w, vsig, u, du, cn1, cn2):
    dtv = cn1 * (w / vsig).abs()
    dte = cn2 * (u / du).abs()
    tau = 1.0 / (1.0 / dtv + 1.0 / dte)
    return tau.min()


def step(state: dict, p: dict):
    """One step.  state: x (N,3), v (N,3), u, a (N,3), du, dt (0-d), m, mu, w
    (previous ranges, used only as the solver's start).  Returns the new state
    dict plus 'rho', 'P', 'phi' diagnostics."""
    x, v, u, a, du, dt = state["x"], state["v"], state["u"], state["a"], state["du"], state["dt"]
    m, mu = state["m"], state["mu"]
    dth = 0.5 * dt
    x1 = x + v * dt
    vp = v + a * dth
    up = u + du * dth
    w = solve_h(x1, state["w"].detach(), p["n_target"], rel_err=p.get("h_tol", 1e-12))
    rho, div, curl, om, ps = density(x1, vp, m, w)
    P = pressure(rho, up, mu, p["eos_mode"], p["gamma"])
    ah, du1, vsig = hydro(x1, vp, m, w, rho, P, div, curl, om, ps, p)
    g, phi = gravity_plummer(x1, m, p["eps"], p.get("G", 1.0))
    a1 = ah + g
    dt1 = timestep(w, vsig, up, du1, p["cn1"], p["cn2"])
    f = 0.5 * dt1 + dth
    v1 = v + a1 * f
    u1 = u + du1 * f
    return {"x": x1, "v": v1, "u": u1, "a": a1, "du": du1, "dt": dt1, "m": m, "mu": mu, "w": w, "rho": rho,
            "P": P, "phi": phi}


def default_params(**kw):
    p = dict(n_target=50.0, gamma=5.0 / 3.0, alpha=1.0, beta=2.0, eos_mode=1, eps=0.01, use_psi=0, cn1=0.3,
             cn2=0.2, G=1.0)
    p.update(kw)
    return p


def state_from_ic(ic: dict, device="cpu", dtype=torch.float64):
    t = lambda k: torch.as_tensor(ic[k], dtype=dtype, device=device)
    x = torch.stack([t("x"), t("y"), t("z")], 1)
    v = torch.stack([t("vx"), t("vy"), t("vz")], 1)
    n = x.shape[0]
    z3 = torch.zeros(n, 3, dtype=dtype, device=device)
    return {"x": x, "v": v, "u": t("u"), "a": z3.clone(), "du": torch.zeros(n, dtype=dtype, device=device),
            "dt": torch.tensor(float(ic.get("dt", 0.0)), dtype=dtype, device=device), "m": t("m"), "mu": t("mu"),
            "w": t("range")}


def loss_ke_density(state: dict, probes):
    """Kinetic energy plus the mean density at the probe particles."""
    ke = 0.5 * (state["m"] * (state["v"] ** 2).sum(1)).sum()
    return ke + state["rho"][probes].mean()
